"""Device Pfaffian stage (RealPfStage, sampling/stage.rs:56-129) through the C ABI: a
host-driven chain of hops, exchanges, accepts and recomputes replayed on the device and by
the oracle's CPU stage with the same candidate configurations (teacher forcing)."""
import numpy as np
import pytest

import oracle_lib as ol
import stage_moves as sm
from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu


def engine(tmp_path, name, **over):
    lat = lattice()
    cfg = dict(lat.CONFIGS[name])
    cfg.update(over)
    nl, init, _ = lat.write_inputs(str(tmp_path / name), **cfg)
    return nl, mvmc().Engine(nl, init, walkers=1, precision=64, seed=1)


@pytest.mark.parametrize("name,over", [("chain16", {}), ("square8", {}), ("square8", {"tp": -0.2, "n_up": 28})])
def test_device_stage_replay_matches_oracle(tmp_path, name, over):
    nl, eng = engine(tmp_path, name, **over)
    d = eng.dims
    ns, ne, nqp = d["nsite"], d["ne"], d["nqp"]
    n = 2 * ne
    params = eng.parameters()
    st = mvmc().Stage(eng)
    rng = np.random.default_rng(5)
    idx0 = sm.random_configuration(rng, ns, ne)
    ops, seq, _ = sm.random_sequence(rng, idx0, ns, ne, 120)
    ref, ref_inv = ol.stage_replay(nl, params, idx0, ops, seq, nqp, n)
    rc, pf0 = st.begin(idx0)
    assert rc == 0
    last = None
    for k, (op, cand) in enumerate(zip(ops, seq)):
        code, ma, sa, mb, sb, ra, rb = (int(v) for v in op)
        if code == sm.PROPOSE_HOP:
            got = last = st.propose_hop(cand, ma, sa)
        elif code == sm.ACCEPT_HOP:
            st.accept_hop(cand, ma, sa, last)
            got = st.state()[0]
        elif code == sm.PROPOSE_EX:
            got = last = st.propose_exchange(cand, ma, sa, mb, sb)
        elif code == sm.ACCEPT_EX:
            st.accept_exchange(cand, ma, sa, mb, sb, ra, rb)
            got = st.state()[0]
        else:
            rc, got = st.recompute(cand)
            assert rc == 0
        scale = np.abs(ref[k]).max()
        assert np.allclose(got, ref[k], rtol=1e-9, atol=1e-11 * scale), (k, code)
    _, inv = st.state()
    assert np.allclose(inv, ref_inv, rtol=1e-8, atol=1e-10 * np.abs(ref_inv).max())
    st.close()
    eng.close()


def test_device_stage_rejects_bad_slots_and_sites(tmp_path):
    _, eng = engine(tmp_path, "chain16")
    st = mvmc().Stage(eng)
    ns, ne = eng.dims["nsite"], eng.dims["ne"]
    idx = sm.random_configuration(np.random.default_rng(0), ns, ne)
    assert st.begin(idx)[0] == 0
    with pytest.raises(RuntimeError, match="status -"):
        st.propose_hop(idx, ne, 0)
    bad = idx.copy()
    bad[0] = ns
    with pytest.raises(RuntimeError, match="out of range"):
        st.propose_hop(bad, 0, 0)
    with pytest.raises(RuntimeError):
        st.propose_exchange(idx, 0, 0, 0, 0)
    st.close()
    eng.close()
