"""Device engine parity: resident sampler, measurement and SR-CG against the native C
golden vectors and the oracle, through the C ABI."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import mvmc, read_triples

pytestmark = pytest.mark.gpu
G = ol.GOLDEN


def physcal_engine(precision=64):
    d = os.path.join(G, "physcal_hubbard_chain_real")
    m = mvmc()
    eng = m.Engine(os.path.join(d, "inputs", "namelist.def"), walkers=1, precision=precision, seed=1)
    p = read_triples(os.path.join(d, "zqp_opt.dat"), eng.dims["npara"])
    nproj = eng.dims["nproj"]
    f = p[nproj:]
    p[nproj:] = f * (4.0 / np.abs(f).max())  # sync_modified_parameter: max |f| = 4
    eng.set_parameters(p)
    return d, eng


def read_state(path):
    out = {}
    for line in open(path):
        parts = line.split()
        out[parts[0]] = [int(v) for v in parts[1:]]
    return out


def test_device_sampler_reproduces_native_c_trajectory():
    """Every saved configuration, projection counter, C Counter[0..6] and the draw count
    of two sample blocks of the native C sampler, from the device-resident sampler."""
    d, eng = physcal_engine()
    for b, idx in enumerate((7, 8)):
        eng.sample()
        got = eng.samples()
        ref = read_state(os.path.join(d, "native-state", f"state_dump_{b:03d}.txt"))
        assert got["ele_idx"].tolist() == ref["ele_idx"]
        assert got["ele_cfg"].tolist() == ref["ele_cfg"]
        assert got["ele_num"].tolist() == ref["ele_num"]
        assert got["proj_cnt"].tolist() == ref["ele_proj_cnt"]
        assert got["counter"].tolist() == ref["counter"][:6]
        assert int(got["draws"][0]) == ref["draws"][0]
        e, _, _ = eng.measure()
        row = open(os.path.join(d, "expected", f"zvo_out_{idx:03d}.dat")).read().split()
        assert abs(e[1] - float(row[0])) <= 1e-12 * abs(float(row[0]))
        assert abs(e[2] - float(row[2])) <= 1e-12 * abs(float(row[2]))
    assert eng.status() == 0


def test_device_step1_sr_operands_match_native_c():
    d = os.path.join(G, "sr_operands_hubbard")
    eng = mvmc().Engine(os.path.join(d, "inputs", "namelist.def"), walkers=1, precision=64, seed=1)
    eng.sample()
    e, ho, oo = eng.measure()
    ref = {}
    for line in open(os.path.join(d, "hubbard-cg-store0.txt")):
        if line.startswith("#"):
            continue
        name, rest = line.split(None, 1)
        ref[name] = ol.hexline(rest)
    assert abs(e[1] - ref["energy"][0]) <= 1e-12 * abs(ref["energy"][0])
    for name, got in (("ho", ho), ("oo", oo)):
        r = ref[name]
        assert np.all(np.abs(got[: len(r)] - r) <= 1e-14 + 1e-13 * np.abs(r)), name
    store = eng.o_store()
    r = ref["o"]
    assert np.all(np.abs(store[-1, : len(r)] - r) <= 1e-14 + 1e-13 * np.abs(r))


@pytest.mark.parametrize("walkers", [1, 3, 8])
def test_multiwalker_step1_matches_oracle(walkers):
    """W chains seeded RndSeed + w: configurations exact, operands within 1e-12."""
    nl = os.path.join(G, "sr_operands_hubbard", "inputs", "namelist.def")
    dims, ref = ol.opt_step1_walkers(nl, walkers, seed=7)
    eng = mvmc().Engine(nl, walkers=walkers, precision=64, seed=7)
    eng.sample()
    got = eng.samples()
    assert got["ele_idx"].tolist() == ref["ele_idx"].tolist()
    assert got["proj_cnt"].tolist() == ref["proj_cnt"].tolist()
    assert got["counter"].tolist() == ref["counter"].tolist()
    assert got["draws"].tolist() == ref["draws"].tolist()
    e, ho, oo = eng.measure()
    assert np.allclose(e, ref["energy"], rtol=1e-12, atol=1e-13)
    assert np.allclose(ho, ref["ho"], rtol=1e-12, atol=1e-13)
    assert np.allclose(oo, ref["oo"], rtol=1e-12, atol=1e-13)
    assert np.allclose(eng.o_store(), ref["ostore"], rtol=1e-11, atol=1e-12)


def read_cg_fixture(path):
    lines = [l.rstrip("\n") for l in open(path) if not l.startswith("#")]
    n, samples, _ = (int(v) for v in lines[0].split())
    mean, diag, real = ol.hexline(lines[1]), ol.hexline(lines[2]), ol.hexline(lines[3])
    g = ol.hexline(lines[5])
    limits = []
    for k in range(7, len(lines), 3):
        head = lines[k].split(" ", 2)
        limits.append((int(head[0]), int(head[1]), ol.hexline(head[2])))
    return n, samples, mean, diag, real, g, limits


@pytest.mark.parametrize("name,diag_scale", [("real.txt", False), ("real_diag_scale.txt", True)])
def test_device_cg_recurrence_matches_native_c(name, diag_scale):
    n, samples, mean, diag, real, g, limits = read_cg_fixture(os.path.join(G, "sr_cg", name))
    m = mvmc()
    for limit, status, x_ref in limits:
        st, x = m.cg_solve(real, mean, diag, g, 1.0 / samples, 1e-5, 0.0, limit, diag_scale)
        assert st == status, limit
        if limit <= 5:
            assert np.allclose(x, x_ref, rtol=1e-8, atol=1e-12 * np.abs(x_ref).max()), limit


def test_device_cg_matches_oracle_on_random_operands():
    rng = np.random.default_rng(5)
    ns, na = 300, 40
    smp = rng.normal(size=(ns, na))
    mean = smp.mean(axis=0)
    diag = (smp * smp).mean(axis=0) - mean * mean
    g = rng.normal(size=na)
    st, x = mvmc().cg_solve(smp, mean, diag, g, 1.0 / ns, 0.02, 1e-10, na)
    ost, ox, _ = ol.cg_fixed(mean, diag, smp.ravel(), g, 1.0 / ns, 0.02, 1e-10, na)
    assert st == ost
    assert np.allclose(x, ox, rtol=1e-9, atol=1e-12)


def cg_inputs(tmp_path, **overrides):
    """Copy the Hubbard-chain inputs with the modpara overrides (NSRCG 1 selects SR-CG)."""
    import shutil
    src = os.path.join(G, "sr_operands_hubbard", "inputs")
    dst = tmp_path / "inputs"
    shutil.copytree(src, dst)
    keys = {"NSRCG": "1", "NSRCGAbortOnFail": "0", **{k: str(v) for k, v in overrides.items()}}
    lines = open(dst / "modpara.def").read().splitlines()
    for k, v in keys.items():
        hit = [i for i, l in enumerate(lines) if l.split()[:1] == [k]]
        if hit:
            lines[hit[0]] = f"{k} {v}"
        else:
            lines.append(f"{k} {v}")
    (dst / "modpara.def").write_text("\n".join(lines) + "\n")
    return str(dst / "namelist.def")


def read_out(path):
    return np.array([[float(v) for v in line.split()] for line in open(path)])


@pytest.mark.parametrize("c_order", [1, 0])
def test_full_optimisation_matches_oracle_zvo_out(tmp_path, c_order):
    """Ten SR steps (sample → measure → SR-CG → sync) with 2 chains of the Hubbard-chain
    example. C-order parity mode: every zvo_out.dat energy within 1e-8 relative of the oracle
    run and the SRinfo rows equal. Throughput kernels (Gauss–Jordan inverse, parallel sums,
    FMA): step 1 within 1e-12 and every step within 1e-6, the envelope that any reordering of
    the SR sums opens (the CG iterate of a step carries the rounding of its operands: in the
    oracle itself, reversing the order of one dot product of the CG product moves later
    energies by 1e-8 … 1e-6)."""
    # a converging CG (tol 1e-8 reached in ~27 iterations)
    nl = cg_inputs(tmp_path, NSROptCGMaxIter=200, DSROptCGTol="1e-8")
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gdir.mkdir()
    odir.mkdir()
    if c_order:
        with ol.fixed_exp_mode():
            ol.run_opt(nl, str(odir), walkers=2, nsteps=10, seed=3)
    else:
        ol.run_opt(nl, str(odir), walkers=2, nsteps=10, seed=3)
    mvmc().run_opt(nl, str(gdir), nsteps=10, walkers=2, precision=64, seed=3, c_order=c_order)
    a = read_out(gdir / "zvo_out.dat")
    b = read_out(odir / "zvo_out.dat")
    assert a.shape == b.shape == (10, 6)
    rel = np.abs(a[:, 0] - b[:, 0]) / np.abs(b[:, 0])
    assert rel[0] <= 1e-12
    assert np.all(rel <= (1e-8 if c_order else 1e-6)), rel.tolist()
    va = read_out(gdir / "zvo_var.dat")
    vb = read_out(odir / "zvo_var.dat")
    # parameters after each step, relative to the largest parameter of the step
    scale = np.abs(vb).max(axis=1, keepdims=True)
    assert np.all(np.abs(va - vb) <= (1e-8 if c_order else 1e-6) * scale)
    for name in ("zqp_opt.dat", "zvo_SRinfo.dat", "zqp_orbital_opt.dat"):
        assert (gdir / name).exists() and (odir / name).exists()
    sa = [l.split() for l in open(gdir / "zvo_SRinfo.dat").read().splitlines()[1:]]
    sb = [l.split() for l in open(odir / "zvo_SRinfo.dat").read().splitlines()[1:]]
    assert [r[:4] for r in sa] == [r[:4] for r in sb]  # NPara, active size, cuts
    assert all(int(r[-1]) >= 0 for r in sa)  # CG converged at every step


def chain16_inputs(tmp_path):
    from mvmc_lib import lattice
    lat = lattice()
    return lat.write_inputs(str(tmp_path / "in"), **dict(lat.CONFIGS["chain16"]))


def test_c_order_step1_operands_bitwise_equal_the_oracle(tmp_path):
    """C-order parity mode on the 1D chain L = 16 (256 chains): the saved configurations,
    every row of the SR sample matrix, HO, <O>, <O^2> and the energy sums equal the oracle's
    (with the same fixed exp in the projection ratios) bit for bit: pfapack LTL inverse,
    serial sums, no FMA."""
    nl, init, _ = chain16_inputs(tmp_path)
    W = 256
    with ol.fixed_exp_mode():
        dims, ref = ol.opt_step1_walkers(nl, W, seed=12345, initial_def=init)
    eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=12345, c_order=1)
    eng.sample()
    assert eng.samples()["ele_idx"].tolist() == ref["ele_idx"].tolist()
    e, ho, oo = eng.measure()
    store = eng.o_store()
    assert np.array_equal(store, ref["ostore"]), np.abs(store - ref["ostore"]).max()
    assert np.array_equal(e, ref["energy"]), (e - ref["energy"]).tolist()
    assert np.array_equal(ho, ref["ho"])
    assert np.array_equal(oo, ref["oo"])
    eng.close()


def test_chain16_full_run_gate_zvo_out_1e8(tmp_path):
    """The full-run parity gate on the 1D Hubbard chain L = 16 (t = 1, U = 4, half filling,
    f with translation symmetry, Gutzwiller and distance Jastrow, parameters uniform
    [-0.05, 0.05] from the seed): 256 chains, NVMCInterval 16, ten SR-CG steps
    (DSROptRedCut 1e-8, DSROptStepDt 0.02), RndSeed 12345, in the C-order parity mode.
    Every zvo_out.dat energy within 1e-8 relative of the oracle run on the same inputs (the
    reference's own 10-step gate, crates/mvmc-core/tests/phase5_zvo_gate_hubbard.rs:19-80),
    the SRinfo rows (active sets, S diagonal extremes, largest update, CG iterations) equal."""
    nl, init, _ = chain16_inputs(tmp_path)
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gdir.mkdir()
    odir.mkdir()
    with ol.fixed_exp_mode():
        ol.run_opt(nl, str(odir), walkers=256, nsteps=10, seed=12345, initial_def=init)
    mvmc().run_opt(nl, str(gdir), initial_def=init, nsteps=10, walkers=256, precision=64, seed=12345, c_order=1)
    a = read_out(gdir / "zvo_out.dat")
    b = read_out(odir / "zvo_out.dat")
    assert a.shape == b.shape == (10, 6)
    rel = np.abs(a[:, 0] - b[:, 0]) / np.abs(b[:, 0])
    assert np.all(rel <= 1e-8), f"relative energy deviation per step: {rel.tolist()}"
    sa = [l.split() for l in open(gdir / "zvo_SRinfo.dat").read().splitlines()[1:]]
    sb = [l.split() for l in open(odir / "zvo_SRinfo.dat").read().splitlines()[1:]]
    assert sa == sb


@pytest.mark.parametrize("ex_path", [0, 1, 2])
def test_interaction_terms_and_update_paths_match_oracle(tmp_path, ex_path):
    """1D L16 with CoulombInter and Hund terms beside U, under each NExUpdatePath (0: hops
    only, 1: hops and exchanges, 2: exchanges only): four chains' configurations, counters
    and draw counts exact, energies and operands within 1e-12 of the oracle."""
    from mvmc_lib import lattice
    lat = lattice()
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), lx=16, U=4.0, V=1.5, J_hund=0.7, ex_path=ex_path,
                                   warmup=4, samples=3, interval=2)
    W = 4
    dims, ref = ol.opt_step1_walkers(nl, W, seed=7, initial_def=init)
    eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=7)
    eng.sample()
    got = eng.samples()
    assert got["ele_idx"].tolist() == ref["ele_idx"].tolist()
    assert got["counter"].tolist() == ref["counter"].tolist()
    assert got["draws"].tolist() == ref["draws"].tolist()
    c = got["counter"].reshape(W, 6).sum(axis=0)
    assert (c[0] > 0) == (ex_path != 2) and (c[2] > 0) == (ex_path != 0)
    e, ho, oo = eng.measure()
    assert np.allclose(e, ref["energy"], rtol=1e-12, atol=1e-13)
    assert np.allclose(ho, ref["ho"], rtol=1e-12, atol=1e-13)
    assert np.allclose(oo, ref["oo"], rtol=1e-12, atol=1e-13)
    eng.close()
