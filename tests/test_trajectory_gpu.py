"""Trajectory-level parity on the 2D 8×8 model with eight QP planes (translation and spin
projection, NQP = 8; the batched-sampler benchmark's model) under the C refresh rule:
the device FP64 sampler against the oracle chain by chain, and both against a long-double
shadow of the same chain (oracle_trace_chain: the oracle's chain with its Pfaffians and
inverses carried in long double by the same algorithms, teacher-forced on the FP64
decisions)."""
import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu

BLOCKS = 5  # the first SR step: 4 warm-up blocks + 1 sample block of 64 sweeps


def square8_every_block_saved(tmp_path):
    """The square8 inputs with every block of the first SR step saved (warm-up 0, five
    samples): the chain is the same as with four warm-up blocks and one sample."""
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg.update(warmup=0, samples=BLOCKS)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
    return nl, init


def test_square8_trajectories_equal_the_oracle(tmp_path):
    """8 chains (seeds 12345 + w), 5 blocks of 64 sweeps (4096 proposals per block): every
    block-end configuration, projection counter, proposal/accept counter and SFMT draw count
    of the device FP64 sampler equals the oracle's."""
    nl, init = square8_every_block_saved(tmp_path)
    W = 8
    _, ref = ol.opt_step1_walkers(nl, W, seed=12345, initial_def=init)
    eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=12345)
    eng.sample()
    got = eng.samples()
    for key in ("ele_idx", "proj_cnt", "counter", "draws"):
        assert got[key].tolist() == ref[key].tolist(), key
    eng.close()


def test_square8_device_log_weights_within_the_oracle_error_of_long_double(tmp_path):
    """Walker 0 of the same run (5 blocks, 20480 proposals, ~100 refreshes): the oracle's
    stage operations replayed on the device stage (mvmc_b200_stage_*, FP64, teacher-forced).
    Against the long-double shadow, the device's Metropolis log-weights
    2(Δln P + ln|IP'| − ln|IP|) are as accurate as the oracle's (max error ≤ 4× the oracle's),
    no device or oracle decision differs from the long-double one, and the device's ln|IP|
    drift at a refresh is at most 4× the oracle's."""
    nl, init = square8_every_block_saved(tmp_path)
    idx0, ops, cands, rec = ol.trace_chain(nl, 0, blocks=BLOCKS, max_ops=60000, seed=12345, initial_def=init)
    qpw = ol.qp_weights(nl)
    eng = mvmc().Engine(nl, init, walkers=1, precision=64, seed=12345)
    st = mvmc().Stage(eng)

    def lip_of(pf):
        return float(np.log(abs(np.dot(qpw, pf))))

    rc, pf0 = st.begin(idx0)
    assert rc == 0
    lip, lipn = lip_of(pf0), None
    lw_dev, rows, drift_dev = [], [], 0.0
    for k in range(len(ops)):
        code, ma, sa, mb, sb, ra, rb = (int(v) for v in ops[k])
        if code in (0, 2):
            pfn = st.propose_hop(cands[k], ma, sa) if code == 0 else st.propose_exchange(cands[k], ma, sa, mb, sb)
            lipn = lip_of(pfn)
            lw_dev.append(2.0 * ((rec[k, 0] + lipn) - lip))
            rows.append(k)
        elif code == 1:
            st.accept_hop(cands[k], ma, sa, None)
            lip = lipn
        elif code == 3:
            st.accept_exchange(cands[k], ma, sa, mb, sb, ra, rb)
            lip = lipn
        else:
            rc, pf = st.recompute(cands[k])
            assert rc == 0
            fresh = lip_of(pf)
            drift_dev = max(drift_dev, abs(lip - fresh))
            lip = fresh
    st.close()
    eng.close()
    r = rec[rows]
    u, lw_orc, lw_ld, lw_dev = r[:, 1], r[:, 2], r[:, 3], np.array(lw_dev)
    assert len(rows) == BLOCKS * 64 * 64
    acc_ld = np.exp(lw_ld) > u
    assert np.array_equal(np.exp(lw_orc) > u, acc_ld)
    assert np.array_equal(np.exp(lw_dev) > u, acc_ld)
    err_orc, err_dev = np.abs(lw_orc - lw_ld).max(), np.abs(lw_dev - lw_ld).max()
    assert err_dev <= 4.0 * err_orc, (err_dev, err_orc)
    refresh = rec[ops[:, 0] == 4]
    drift_orc = np.abs(refresh[:, 0] - refresh[:, 2]).max()
    assert drift_dev <= 4.0 * drift_orc + 1e-12, (drift_dev, drift_orc)


def read_out(path):
    return np.array([[float(v) for v in line.split()] for line in open(path)])


def test_square8_ten_step_gate_zvo_out_c_order(tmp_path):
    """The 10-step zvo_out.dat gate on the benchmark model (2D 8×8, NQP = 8; 8 chains,
    RndSeed 12345, ten SR-CG steps) in the C-order parity mode: the device sampler, the
    C-order measurement and CG against the oracle with the same exponential in the
    projection ratios. Every energy within 1e-8 relative (observed: equal bit for bit, also
    with 16 chains) and every SRinfo row equal. The throughput kernels leave this envelope
    after the first step (2e-7 at step 2): the SR-CG solution carries the summation order of
    the measurement and CG sums."""
    lat = lattice()
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **dict(lat.CONFIGS["square8"]))
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gdir.mkdir()
    odir.mkdir()
    with ol.fixed_exp_mode():
        ol.run_opt(nl, str(odir), walkers=8, nsteps=10, seed=12345, initial_def=init)
    mvmc().run_opt(nl, str(gdir), initial_def=init, nsteps=10, walkers=8, precision=64, seed=12345, c_order=1)
    a, b = read_out(gdir / "zvo_out.dat"), read_out(odir / "zvo_out.dat")
    assert a.shape == b.shape == (10, 6)
    rel = np.abs(a[:, 0] - b[:, 0]) / np.abs(b[:, 0])
    assert np.all(rel <= 1e-8), rel.tolist()
    sa = open(gdir / "zvo_SRinfo.dat").read().splitlines()[1:]
    sb = open(odir / "zvo_SRinfo.dat").read().splitlines()[1:]
    assert sa == sb
