"""Pins the oracle (the CPU checker) to the reference's own golden vectors.

Every fixture under tests/golden/ is output of the native C mVMC 1.4.0 program or of
the C SFMT library, copied from the reference by tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as ol

G = ol.GOLDEN


def test_sfmt_first_words_match_c_library():
    gold = json.load(open(os.path.join(G, "sfmt_first8.json")))
    assert len(gold) == 6
    for seed, words in gold.items():
        assert ol.sfmt_words(int(seed), 8) == words, seed


def read_pfapack(path):
    vals = [float(l) for l in open(path) if l.strip() and not l.startswith("#") and " " not in l.strip()]
    n = int(round(len(vals) ** 0.5))
    return np.array(vals).reshape(n, n), n


@pytest.mark.parametrize("name", sorted(os.listdir(os.path.join(G, "pfapack"))))
def test_pfaffian_identities_on_reference_matrices(name):
    # crates/pfapack/tests/fixed_matrix_identities.rs: Pf^2 = det, inverse residual <= 64 eps.
    x, n = read_pfapack(os.path.join(G, "pfapack", name))
    assert np.allclose(x, -x.T)
    pf, inv, st = ol.pfinv_batch(x.T.ravel(), n, 1)
    assert st[0] == 0
    xi = inv.reshape(n, n).T
    sign, logdet = np.linalg.slogdet(x)
    assert sign > 0
    assert abs(2 * np.log(abs(pf[0])) - logdet) <= n * 1e-13
    eps = np.finfo(float).eps
    resid = np.abs(xi @ x - np.eye(n)).max() / (np.abs(x).max() * np.abs(xi).max())
    assert resid <= 64 * eps * n


def test_pfaffian_zero_pivot_reports_row():
    x = np.zeros((4, 4))
    x[0, 1], x[1, 0] = 1.0, -1.0  # rank 2: the elimination meets a zero column
    pf, inv, st = ol.pfinv_batch(x.T.ravel(), 4, 1)
    assert st[0] > 0


def read_state(path):
    out = {}
    for line in open(path):
        p = line.split()
        out[p[0]] = p[1:]
    return out


def test_sampler_reproduces_native_c_trajectory():
    """Every saved configuration, projection counter, C Counter[0..6], draw count and
    the next 624 SFMT words of two sample blocks of the native C sampler."""
    d = os.path.join(G, "physcal_hubbard_chain_real")
    dims, out = ol.physcal_samples(os.path.join(d, "inputs", "namelist.def"),
                                   os.path.join(d, "zqp_opt.dat"), seed=1)
    n, ns2, npj, S = 2 * dims["ne"], 2 * dims["nsite"], dims["nproj"], dims["nvmc_sample"]
    for b in range(dims["data_qty_smp"]):
        ref = read_state(os.path.join(d, "native-state", f"state_dump_{b:03d}.txt"))
        for key, name, width in [("ele_idx", "ele_idx", n), ("ele_cfg", "ele_cfg", ns2),
                                 ("ele_num", "ele_num", ns2), ("proj_cnt", "ele_proj_cnt", npj)]:
            got = out[key][b * S * width:(b + 1) * S * width]
            assert got.tolist() == [int(v) for v in ref[name]], (b, key)
        assert out["counter"][b * 6:(b + 1) * 6].tolist() == [int(v) for v in ref["counter"][:6]]
        assert int(out["draws"][b]) == int(ref["draws"][0])
        assert out["next624"][b * 624:(b + 1) * 624].tolist() == [int(v) for v in ref["next624"]]


def test_physcal_energy_matches_native_c_zvo_out():
    d = os.path.join(G, "physcal_hubbard_chain_real")
    dims, out = ol.physcal_samples(os.path.join(d, "inputs", "namelist.def"),
                                   os.path.join(d, "zqp_opt.dat"), seed=1)
    for b, idx in enumerate((7, 8)):
        row = open(os.path.join(d, "expected", f"zvo_out_{idx:03d}.dat")).read().split()
        etot, etot2 = float(row[0]), float(row[2])
        assert abs(out["energies"][2 * b] - etot) <= 1e-12 * abs(etot)
        assert abs(out["energies"][2 * b + 1] - etot2) <= 1e-12 * abs(etot2)


def test_step1_sr_operands_match_native_c():
    """crates/mvmc-core/tests/c_sr_operands_358.rs: ABS 1e-14 / REL 1e-13, energy 1e-12."""
    d = os.path.join(G, "sr_operands_hubbard")
    got = ol.step1_operands(os.path.join(d, "inputs", "namelist.def"), cg=1, store=0, seed=1)
    ref = {}
    for line in open(os.path.join(d, "hubbard-cg-store0.txt")):
        if line.startswith("#"):
            continue
        name, rest = line.split(None, 1)
        ref[name] = ol.hexline(rest)
    assert abs(got["energy"][0] - ref["energy"][0]) <= 1e-12 * (1 + abs(ref["energy"][0]))
    for name in ("ho", "oo", "o"):
        r = ref[name]
        a = got[name][: len(r)]
        assert np.all(np.abs(a - r) <= 1e-14 + 1e-13 * np.abs(r)), name


def read_cg_fixture(path):
    lines = [l.rstrip("\n") for l in open(path) if not l.startswith("#")]
    n, samples, cplx = (int(v) for v in lines[0].split())
    assert cplx == 0
    mean, diag, real = ol.hexline(lines[1]), ol.hexline(lines[2]), ol.hexline(lines[3])
    g, expected_apply = ol.hexline(lines[5]), ol.hexline(lines[6])
    limits = []
    k = 7
    while k + 2 < len(lines) + 1 and k < len(lines):
        head = lines[k].split(" ", 2)
        limits.append((int(head[0]), int(head[1]), ol.hexline(head[2])))
        k += 3
    return n, samples, mean, diag, real, g, expected_apply, limits


@pytest.mark.parametrize("name,diag_scale", [("real.txt", False), ("real_diag_scale.txt", True)])
def test_cg_recurrence_matches_native_c(name, diag_scale):
    """C StochasticOptCG on fixed operands (tol 0, shift 1e-5): statuses exact,
    S·g within the two-GEMV rounding budget, iterates within 1e-8 relative for the
    first limits (CG amplifies roundoff after the residual drops)."""
    n, samples, mean, diag, real, g, expected_apply, limits = read_cg_fixture(
        os.path.join(G, "sr_cg", name))
    _, _, z = ol.cg_fixed(mean, diag, real, g, 1.0 / samples, 1e-5, 0.0, 1, diag_scale, True)
    budget = 8.0 * (n + samples) * np.finfo(float).eps
    assert np.all(np.abs(z - expected_apply) <= budget + budget * np.abs(expected_apply))
    for limit, status, x_ref in limits:
        st, x, _ = ol.cg_fixed(mean, diag, real, g, 1.0 / samples, 1e-5, 0.0, limit, diag_scale)
        assert st == status, limit
        if limit <= 5:
            assert np.allclose(x, x_ref, rtol=1e-8, atol=1e-12 * np.abs(x_ref).max()), limit


def test_cholesky_solve_matches_numpy_and_reports_pivot():
    rng = np.random.default_rng(4)
    m = rng.normal(size=(40, 40))
    a = m @ m.T + 40 * np.eye(40)
    b = rng.normal(size=40)
    info, x = ol.cholesky_solve(a, b)
    assert info == 0
    assert np.allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-14)
    bad = a.copy()
    bad[5, 5] = -1.0
    info, _ = ol.cholesky_solve(bad, b)
    assert info == 6


def test_direct_sr_optimisation_runs_and_updates(tmp_path):
    """NSRCG 0 (the reference example's default): Gram, redundancy cut, S and g, the
    Cholesky solve and the update over three steps; SRinfo rows carry no info column."""
    nl = os.path.join(G, "sr_operands_hubbard", "inputs", "namelist.def")
    ol.run_opt(nl, str(tmp_path), walkers=2, nsteps=3, seed=3)
    rows = np.loadtxt(tmp_path / "zvo_out.dat")
    assert rows.shape[0] == 3 and np.all(np.isfinite(rows))
    info = open(tmp_path / "zvo_SRinfo.dat").read().splitlines()
    assert info[0].split()[-1] == "imax"
    assert len(info) == 4 and all(len(r.split()) == 8 for r in info[1:])


def test_fixed_exp_is_within_one_ulp_of_libm():
    """The exp of the C-order parity mode (Cody–Waite reduction, degree-13 Taylor polynomial,
    exact 2^k scaling) agrees with the platform libm to one ulp over the arguments the
    projection ratios take and at the range ends."""
    import math
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-40, 40, 20000), rng.uniform(-1, 1, 20000),
                         [0.0, -0.0, 1e-300, -1e-300, 700.0, -700.0, -744.0, 709.7]])
    for x in xs:
        a, b = ol.fixed_exp(x), math.exp(x)
        assert abs(a - b) <= math.ulp(b), x
    assert ol.fixed_exp(0.0) == 1.0 and ol.fixed_exp(800.0) == math.inf and ol.fixed_exp(-800.0) == 0.0


def test_fixed_exp_oracle_keeps_its_native_c_pins():
    """With the fixed exp in the local energy the oracle still meets the native C pins:
    PhysCal energies (1e-12) and step-1 SR operands (abs 1e-14 / rel 1e-13)."""
    with ol.fixed_exp_mode():
        test_physcal_energy_matches_native_c_zvo_out()
        test_step1_sr_operands_match_native_c()


def test_square8_fp64_chain_decisions_equal_a_long_double_shadow(tmp_path):
    """The reference algorithm in FP64 on the 2D 8×8 model with eight QP planes (NQP = 8,
    C refresh rule), walker 0 of the first SR step (5 blocks of 64 sweeps, 20480
    proposals), against a long-double shadow of the same chain (same proposals and refresh
    points, Pfaffians and inverses carried in long double by the same algorithms): every
    Metropolis decision equals the long-double one; the log-weights agree within 1e-3
    (observed 4e-5), the FP64 recomputation of ln|IP| within 1e-12, the FP64 rank-2 drift
    before a refresh stays below 1e-5 and the long-double one below 1e-8."""
    from mvmc_lib import lattice
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg.update(warmup=0, samples=5)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
    idx0, ops, cands, rec = ol.trace_chain(nl, 0, blocks=5, max_ops=60000, seed=12345, initial_def=init)
    prop = (ops[:, 0] == 0) | (ops[:, 0] == 2)
    r = rec[prop]
    assert len(r) == 5 * 64 * 64
    u, lw64, lwld = r[:, 1], r[:, 2], r[:, 3]
    assert np.array_equal(np.exp(lw64) > u, np.exp(lwld) > u)
    assert np.array_equal(r[:, 4] != 0, np.exp(lw64) > u)
    assert np.abs(lw64 - lwld).max() < 1e-3
    rc = rec[ops[:, 0] == 4]
    assert len(rc) > 50
    assert np.abs(rc[:, 1] - rc[:, 2]).max() < 1e-12
    assert np.abs(rc[:, 0] - rc[:, 2]).max() < 1e-5
    assert np.abs(rc[:, 3] - rc[:, 2]).max() < 1e-8
