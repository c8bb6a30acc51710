"""The walker-sharded SR step (mvmc-rs_b200/sharded.py) on the device engine with one rank
(identity reducer) against the engine's own SR-CG on the same samples."""
import os
import sys

import numpy as np
import pytest

from mvmc_lib import ROOT, lattice, mvmc

sys.path.insert(0, os.path.join(ROOT, "mvmc-rs_b200"))
import sharded  # noqa: E402

pytestmark = pytest.mark.gpu


def test_sharded_step_on_one_rank_matches_engine_sr(tmp_path):
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    # a tight CG tolerance (1e-10; below that the C breakdown guard |δ| < 1e-20 is reached
    # first) and a larger diagonal shift: the two recurrences (different summation orders)
    # then agree within 5 % of the bound over several seeds
    cfg.update(interval=2, cg_tol=1e-10, cg_max_iter=2000, sta_del=0.1)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
    # 1024 samples for 162 parameters: with 256 the SR matrix is close enough to singular
    # that the two CG recurrences (different summation orders) end up to 5e-6 apart
    a = mvmc().Engine(nl, init, walkers=1024, precision=64, seed=9)
    b = mvmc().Engine(nl, init, walkers=1024, precision=64, seed=9)
    p0 = a.parameters()
    for eng in (a, b):
        eng.sample()
        eng.measure()
    # same chains, and every reduction of the measurement runs in a fixed order: equal sums
    assert np.array_equal(a.measure_sums(), b.measure_sums())
    b.close()
    # both solves on the same measured O store (the SR matrix is ill-conditioned enough that
    # rounding-level differences of the store move the solution by more than the CG tolerance)
    sinfo = sharded.sr_step(a, lambda x: x)
    db = a.parameters() - p0
    a.set_parameters(p0)
    rc, info = a.sr_cg()
    da = a.parameters() - p0
    assert rc == 0 and info[8] >= 0 and sinfo["info"] >= 0
    assert sinfo["nsmat"] == int(info[1]) and sinfo["opt_cut"] == int(info[2]) and sinfo["diag_cut"] == int(info[3])
    assert np.allclose(db, da, rtol=1e-6, atol=1e-6 * np.abs(da).max())
    a.close()


def test_device_resident_sharded_step_matches_engine_sr(tmp_path):
    """sr_step_device on one rank: the CG vectors stay on the GPU (torch tensors), the local
    product runs on device buffers (mvmc_b200_sr_local_product_device); same update as the
    engine's own SR-CG on the same measured samples within the CG tolerance."""
    import torch
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg.update(interval=2, cg_tol=1e-10, cg_max_iter=2000, sta_del=0.1)
    nl, init, _ = lat.write_inputs(str(tmp_path / "in"), **cfg)
    a = mvmc().Engine(nl, init, walkers=1024, precision=64, seed=9)
    p0 = a.parameters()
    a.sample()
    a.measure()
    stream = torch.cuda.current_stream().cuda_stream
    sinfo = sharded.sr_step_device(a, lambda x: x, lambda t: None, "cuda", stream)
    db = a.parameters() - p0
    a.set_parameters(p0)
    rc, info = a.sr_cg()
    da = a.parameters() - p0
    assert rc == 0 and info[8] >= 0 and sinfo["info"] >= 0 and sinfo["nsmat"] == int(info[1])
    assert np.allclose(db, da, rtol=1e-6, atol=1e-6 * np.abs(da).max())
    a.close()
