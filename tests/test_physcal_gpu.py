"""PhysCal (NVMCCalMode 1) on the device through the C ABI: energies and Green functions
(zvo_cisajs, zvo_cisajscktalt, zvo_cisajscktaltex) against the native C mVMC 1.4.0 outputs
of the reference fixture native_c_physcal_181/hubbard_chain_real on 1, 2 and 4 chains,
and against the oracle on Green lists that reach every branch of the two-body reduction
(general two-hop terms included), on the 1D chain and on the 2D 8×8 model."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import green_term_mix, lattice, mvmc, write_green_lists

pytestmark = pytest.mark.gpu
D = os.path.join(ol.GOLDEN, "physcal_hubbard_chain_real")
NL = os.path.join(D, "inputs", "namelist.def")
ZQP = os.path.join(D, "zqp_opt.dat")


def c_close(got, ref):
    """The reference's bound for this scenario (issue181_native_c_physcal.rs:91-109)."""
    return np.all(np.abs(got - ref) <= np.maximum(1e-13, 1e-10 * np.abs(ref)))


def o_close(got, ref, rtol=1e-11):
    return np.all(np.abs(got - ref) <= rtol * np.maximum(1.0, np.abs(ref)))


@pytest.mark.parametrize("walkers,sub", [(1, "expected"), (2, "expected_mpi2"), (4, "expected_mpi4")])
def test_green_functions_match_native_c(walkers, sub):
    eng = mvmc().Engine(NL, physcal_zqp=ZQP, walkers=walkers, precision=64, seed=1)
    assert eng.green_dims == {"one": 12, "ex": 3, "two": 36, "blocks": 2, "idx_start": 7}
    _, ref = ol.physcal_green(NL, ZQP, 1, walkers)
    for b, idx in enumerate((7, 8)):
        eng.sample()
        e, one, ex, two = eng.measure_green()
        c = ol.read_physcal_expected(os.path.join(D, sub), idx)
        assert c_close(e[1:], c["energy"]), (b, e, c["energy"])
        assert c_close(one, c["one"]) and c_close(ex, c["ex"]) and c_close(two, c["two"])
        assert o_close(e[1:], ref["energy"][b], 1e-13)
        for k, v in (("one", one), ("ex", ex), ("two", two)):
            assert o_close(v, ref[k][b], 1e-13), k
    assert eng.status() == 0
    eng.close()


def test_run_physcal_writes_the_c_files(tmp_path):
    mvmc().run_physcal(NL, ZQP, str(tmp_path), walkers=1, precision=64, seed=1)
    for idx in (7, 8):
        for kind in ("out", "var", "cisajs", "cisajscktalt", "cisajscktaltex"):
            name = f"zvo_{kind}_{idx:03d}.dat"
            got = open(tmp_path / name).read().split("\n")
            ref = open(os.path.join(D, "expected", name)).read().split("\n")
            assert len(got) == len(ref), name
            for a, b in zip(got, ref):
                ta, tb = a.split(), b.split()
                assert len(ta) == len(tb), (name, a, b)
                for x, y in zip(ta, tb):
                    if "e" in y or "." in y:
                        assert abs(float(x) - float(y)) <= max(1e-13, 1e-10 * abs(float(y))), (name, x, y)
                    else:
                        assert x == y, (name, a, b)


@pytest.fixture(params=["0", "1"], ids=["per-term", "dense"])
def one_body_path(request, monkeypatch):
    """The one-body plane sums per term (warp per allowed hop) or as the dense product over
    all (empty site, electron) pairs."""
    monkeypatch.setenv("MVMC_B200_GREEN_DENSE", request.param)
    return request.param


def test_all_two_body_branches_match_oracle_on_the_chain(tmp_path, one_body_path):
    one, two, ex = green_term_mix(6, np.random.default_rng(3))
    nl = write_green_lists(os.path.join(D, "inputs"), str(tmp_path / "in"), one, two, ex)
    W = 3
    g, ref = ol.physcal_green(nl, ZQP, 5, W)
    eng = mvmc().Engine(nl, physcal_zqp=ZQP, walkers=W, precision=64, seed=5)
    assert (eng.green_dims["one"], eng.green_dims["ex"], eng.green_dims["two"]) == (g["one"], g["ex"], g["two"])
    for b in range(g["blocks"]):
        eng.sample()
        e, o1, ox, o2 = eng.measure_green()
        assert o_close(e[1:], ref["energy"][b], 1e-12)
        assert o_close(o1, ref["one"][b]) and o_close(ox, ref["ex"][b]) and o_close(o2, ref["two"][b])
        assert np.count_nonzero(o2) > 50
    eng.close()


def test_green_functions_on_square8_match_oracle(tmp_path, one_body_path):
    """2D 8×8 (n = 64, 8 QP planes): the planes live in shared memory during the
    measurement; 8 chains of 4 samples each."""
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg["interval"] = 1
    nl0, init, dims = lat.write_inputs(str(tmp_path / "base"), **cfg)
    # a PhysCal namelist over the same model, with fixed parameters from initial.def
    rng = np.random.default_rng(9)
    ns = 64
    one = [(int(i), s, int(j), s) for s in (0, 1) for i, j in rng.integers(0, ns, (40, 2))]
    one += [(i, 0, i, 0) for i in range(4)] + [(0, 0, 1, 1)] + [one[3], one[50]]  # repeats too
    _, two, ex = green_term_mix(ns, rng, n_two=120)
    nl = write_green_lists(os.path.dirname(nl0), str(tmp_path / "pc"), one, two, ex[:4])
    with open(os.path.join(os.path.dirname(nl), "modpara.def")) as f:
        text = f.read()
    import re
    text = re.sub(r"NVMCCalMode\s+\d+", "NVMCCalMode 1", text)
    text = re.sub(r"NVMCSample\s+\d+", "NVMCSample 4", text)
    text = re.sub(r"NVMCWarmUp\s+\d+", "NVMCWarmUp 2", text)
    text = re.sub(r"NDataQtySmp\s+\d+", "NDataQtySmp 1", text) if "NDataQtySmp" in text else text + "NDataQtySmp 1\n"
    with open(os.path.join(os.path.dirname(nl), "modpara.def"), "w") as f:
        f.write(text)
    W = 8
    g, ref = ol.physcal_green(nl, init, 2, W)
    eng = mvmc().Engine(nl, physcal_zqp=init, walkers=W, precision=64, seed=2)
    eng.sample()
    e, o1, ox, o2 = eng.measure_green()
    assert o_close(e[1:], ref["energy"][0], 1e-10)
    assert o_close(o1, ref["one"][0], 1e-10) and o_close(ox, ref["ex"][0], 1e-10)
    assert o_close(o2, ref["two"][0], 1e-10)
    eng.close()


def test_correlation_lists_on_square8_match_oracle(tmp_path, one_body_path):
    """The bench workload's lists (every same-spin one-body pair, every density-density
    pair) on 8 chains: the dense product path by default."""
    lat = lattice()
    cfg = dict(lat.CONFIGS["physcal8"])
    cfg.update(samples=2, warmup=2)
    nl, init, dims = lat.write_inputs(str(tmp_path / "in"), **cfg)
    W = 8
    g, ref = ol.physcal_green(nl, init, 4, W)
    eng = mvmc().Engine(nl, physcal_zqp=init, walkers=W, precision=64, seed=4)
    assert eng.green_dims["one"] == 8192 and eng.green_dims["two"] == 16384
    eng.sample()
    e, o1, ox, o2 = eng.measure_green()
    assert o_close(e[1:], ref["energy"][0], 1e-10)
    assert o_close(o1, ref["one"][0], 1e-10) and o_close(o2, ref["two"][0], 1e-10)
    eng.close()
