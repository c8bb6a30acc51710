"""Adjoint log-derivative rows O_k = d ln|Psi| / d alpha_k (read from the FP64 inverse of
each saved sample and written straight into the SR sample matrix) on 2D square-lattice
Hubbard models with spin and translation projection:

* against central finite differences of ln|Psi| (step 1e-6, FP64) on 64 random
  (sample, parameter) pairs — the parameters are shifted on the device and the same saved
  configurations re-measured;
* against the oracle's SROptO rows on a 32-walker ensemble with identical configurations
  (the reference's calculate_oo_store_real rows, observables.rs:297).
"""
import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu


def inputs(tmp_path, name, interval, **over):
    lat = lattice()
    cfg = dict(lat.CONFIGS[name])
    cfg["interval"] = interval
    cfg.update(over)
    return lat.write_inputs(str(tmp_path / name), **cfg)


@pytest.mark.parametrize("name,over", [("square8", {}), ("square8", {"tp": -0.2, "n_up": 28}), ("square16", {})])
def test_o_rows_match_central_differences(tmp_path, name, over):
    """64 random (sample, parameter) pairs per model: 2D 8x8 at half filling, 2D 8x8 with
    t' = -0.2 at 56 electrons, and the 2D 16x16 adjoint-check model (t' = -0.2, U = 6,
    112 + 112 electrons, n = 224, full translation symmetry: inverse planes swept as packed
    triangles in shared memory)."""
    nl, init, dims = inputs(tmp_path, name, 2, **over)
    W = 32
    eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=5)
    eng.sample()
    eng.measure()
    o = eng.o_store()
    base = eng.log_amplitudes()
    p0 = eng.parameters()
    npara, nproj = len(p0), eng.dims["nproj"]
    rows = o.shape[0]
    rng = np.random.default_rng(11)
    # 48 pairs on the pair orbitals f_ij, 16 on the Gutzwiller/Jastrow weights
    pairs = [(int(rng.integers(rows)), int(rng.integers(nproj, npara))) for _ in range(48)]
    pairs += [(int(rng.integers(rows)), int(rng.integers(0, nproj))) for _ in range(16)]
    h = 1e-6
    worst = 0.0
    for k in sorted({k for _, k in pairs}):
        p = p0.copy()
        p[k] = p0[k] + h
        eng.set_parameters(p)
        eng.measure()
        lp = eng.log_amplitudes()
        p[k] = p0[k] - h
        eng.set_parameters(p)
        eng.measure()
        lm = eng.log_amplitudes()
        fd = (lp - lm) / (2 * h)
        for r, kk in pairs:
            if kk != k:
                continue
            err = abs(fd[r] - o[r, 1 + k])
            worst = max(worst, err / (1.0 + abs(o[r, 1 + k])))
            assert err <= 1e-6 * (1.0 + abs(o[r, 1 + k])), (r, k, fd[r], o[r, 1 + k])
    # restoring the parameters restores ln|Psi| exactly
    eng.set_parameters(p0)
    eng.measure()
    assert np.array_equal(eng.log_amplitudes(), base)
    eng.close()


@pytest.mark.parametrize("measure", ["packed", "l2"])
def test_o_rows_match_oracle_sroopt_on_32_walkers(tmp_path, monkeypatch, measure):
    """2D 16x16 (t' = -0.2, 112 + 112 electrons, n = 224): every configuration of the 32
    chains equals the oracle's, and so do the SROptO rows — with the planes swept as packed
    triangles in shared memory (default) and in place in L2."""
    if measure == "l2":
        monkeypatch.setenv("MVMC_B200_MEASURE", "l2")
    else:
        monkeypatch.delenv("MVMC_B200_MEASURE", raising=False)
    nl, init, dims = inputs(tmp_path, "square16", 1)
    W = 32
    _, ref = ol.opt_step1_walkers(nl, W, seed=21, initial_def=init)
    eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=21)
    eng.sample()
    got = eng.samples()
    assert got["ele_idx"].tolist() == ref["ele_idx"].tolist()
    e, ho, oo = eng.measure()
    assert np.allclose(e, ref["energy"], rtol=1e-11, atol=1e-12)
    o = eng.o_store()
    assert np.allclose(o, ref["ostore"], rtol=1e-10, atol=1e-11 * np.abs(ref["ostore"]).max())
    assert np.allclose(ho, ref["ho"], rtol=1e-10, atol=1e-11 * np.abs(ref["ho"]).max())
    eng.close()


@pytest.mark.parametrize("name", ["square8", "square16"])
def test_o_rows_are_bitwise_repeatable(tmp_path, name):
    """The same saved samples measured twice give bit-identical O rows, energies and sums:
    every reduction, the Slater derivative included, runs in a fixed order (2D 8x8 with 8
    QP planes in shared memory; 2D 16x16, n = 224, packed triangles)."""
    nl, init, dims = inputs(tmp_path, name, 1)
    eng = mvmc().Engine(nl, init, walkers=64, precision=64, seed=3)
    eng.sample()
    e1, ho1, oo1 = eng.measure()
    o1 = eng.o_store().copy()
    e2, ho2, oo2 = eng.measure()
    o2 = eng.o_store()
    assert np.array_equal(o1, o2)
    assert np.array_equal(e1, e2) and np.array_equal(ho1, ho2) and np.array_equal(oo1, oo2)
    eng.close()
