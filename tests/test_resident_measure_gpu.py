"""The resident measurement (option measure_resident, FP64 path): the sampler stores each
saved sample's Pf and X⁻¹ as it holds them at the save point and the measurement reads
them instead of recomputing them from the configuration (the reference recomputes them,
CalculateMAll per sample). Same chains, same seeds: the measured sums and every row of the
SR sample matrix against the recomputing measurement."""
import numpy as np
import pytest

from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,over,guard,rtol", [
    ("chain16", {}, 0.0, 1e-9),                     # n = 16, planes in shared memory
    ("square16", {"samples": 2}, 0.0, 1e-9),        # n = 224, one plane, packed measurement
    ("square8", {"interval": 4}, 1e-3, 1e-5),       # eight QP planes in L2, refresh guard on
])
def test_resident_measurement_matches_recomputed(tmp_path, name, over, guard, rtol):
    """Energies and O rows within rtol relative of the recomputed measurement: the inverse
    the sampler carries differs from a fresh one by its rank-2 / rank-4 drift (rounding level
    with one plane; with eight projected planes the refresh guard bounds it)."""
    lat = lattice()
    cfg = dict(lat.CONFIGS[name])
    cfg.update(over)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
    W = 64
    out = []
    for resident in (0, 1):
        eng = mvmc().Engine(nl, init, walkers=W, precision=64, seed=11, refresh_guard=guard,
                            measure_resident=resident)
        eng.sample()
        idx = eng.samples()["ele_idx"].copy()
        e, ho, oo = eng.measure()
        out.append((idx, e.copy(), ho.copy(), eng.o_store().copy()))
        eng.close()
    (i0, e0, h0, o0), (i1, e1, h1, o1) = out
    assert np.array_equal(i0, i1)
    assert np.allclose(e1, e0, rtol=rtol, atol=rtol * np.abs(e0).max())
    assert np.allclose(h1, h0, rtol=rtol, atol=rtol * np.abs(h0).max())
    assert np.allclose(o1, o0, rtol=rtol, atol=rtol * np.abs(o0).max())
