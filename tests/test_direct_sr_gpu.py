"""Direct SR (NSRCG 0, the reference example's default) on the device: the Gram of the SR
sample matrix, the Cholesky solve, and full optimisation runs against the oracle."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu
G = ol.GOLDEN


@pytest.mark.parametrize("n,samples", [(7, 3), (163, 300), (333, 1000)])
def test_gram_matches_numpy(n, samples):
    rng = np.random.default_rng(n)
    store = rng.normal(size=(samples, n))
    got = mvmc().gram(store)
    ref = store.T @ store
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert np.array_equal(got, got.T)


@pytest.mark.parametrize("n", [1, 5, 32, 33, 100, 257, 700])
def test_cholesky_solve_matches_oracle_and_numpy(n):
    rng = np.random.default_rng(100 + n)
    m = rng.normal(size=(n, n))
    a = m @ m.T + n * np.eye(n)
    b = rng.normal(size=n)
    rc, x = mvmc().cholesky_solve(a, b)
    assert rc == 0
    info, xo = ol.cholesky_solve(a, b)
    assert info == 0
    ref = np.linalg.solve(a, b)
    assert np.allclose(x, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    assert np.allclose(x, xo, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_cholesky_solve_reports_indefinite_matrix():
    a = np.eye(40)
    a[17, 17] = -2.0
    rc, _ = mvmc().cholesky_solve(a, np.ones(40))
    assert rc == 1


def read_out(path):
    return np.array([[float(v) for v in line.split()] for line in open(path)])


@pytest.mark.parametrize("case", ["hubbard_chain", "square8"])
def test_direct_sr_optimisation_matches_oracle(tmp_path, case):
    """Ten SR steps with the direct solver: energies within 1e-6 of the oracle run (step 1
    within 1e-12), same active sets, parameters close."""
    if case == "hubbard_chain":
        nl, init, steps, W = os.path.join(G, "sr_operands_hubbard", "inputs", "namelist.def"), "", 10, 2
    else:
        lat = lattice()
        cfg = dict(lat.CONFIGS["square8"])
        cfg.update(interval=2, steps=6, nsrcg=0)
        nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
        steps, W = 6, 16
    gdir, odir = tmp_path / "gpu", tmp_path / "oracle"
    gdir.mkdir()
    odir.mkdir()
    ol.run_opt(nl, str(odir), walkers=W, nsteps=steps, seed=3, initial_def=init)
    mvmc().run_opt(nl, str(gdir), initial_def=init, nsteps=steps, walkers=W, precision=64, seed=3)
    a = read_out(gdir / "zvo_out.dat")
    b = read_out(odir / "zvo_out.dat")
    assert a.shape == b.shape == (steps, 6)
    assert abs(a[0, 0] - b[0, 0]) <= 1e-12 * abs(b[0, 0])
    assert np.all(np.abs(a[:, 0] - b[:, 0]) <= 1e-6 * np.abs(b[:, 0]))
    sa = [l.split() for l in open(gdir / "zvo_SRinfo.dat").read().splitlines()]
    sb = [l.split() for l in open(odir / "zvo_SRinfo.dat").read().splitlines()]
    assert sa[0] == sb[0] and sa[0][-1] == "imax"  # direct-mode header: no info column
    assert [r[:4] for r in sa[1:]] == [r[:4] for r in sb[1:]]
    va = read_out(gdir / "zvo_var.dat")
    vb = read_out(odir / "zvo_var.dat")
    scale = np.abs(vb).max(axis=1, keepdims=True)
    assert np.all(np.abs(va - vb) <= 1e-6 * scale)


@pytest.mark.parametrize("sr_precision,bound", [(32, 1e-2), (16, 5e-2)])
def test_direct_sr_through_tensor_core_gram(tmp_path, sr_precision, bound):
    """Direct SR (NSRCG 0) with sr_precision 32 / 16: the active S block from the
    tensor-core Gram of the centred, column-scaled samples (TF32 / BF16 inputs, FP32
    accumulation), the Cholesky solve in FP64. On identical samples (FP64 sampling, same
    seeds) the active set equals the FP64 direct step's and the parameter update is within
    1e-2 (TF32) / 5e-2 (BF16) relative of it."""
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg.update(interval=2, nsrcg=0)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)

    def update(srp):
        eng = mvmc().Engine(nl, init, walkers=1024, precision=64, seed=7, sr_precision=srp)
        p0 = eng.parameters()
        eng.sample()
        eng.measure()
        rc, info = eng.sr_cg()
        dp = eng.parameters() - p0
        eng.close()
        return rc, info, dp

    rc64, info64, d64 = update(64)
    rc, info, d = update(sr_precision)
    assert rc == rc64 == 0
    assert np.array_equal(info[:4], info64[:4]), (info, info64)
    assert np.linalg.norm(d64) > 0
    err = np.linalg.norm(d - d64) / np.linalg.norm(d64)
    assert err <= bound, err
