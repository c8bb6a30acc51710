"""Mixed path (FP32 inverse updates with an FP64 refresh every NRefresh sweeps) against the
plain FP64 path on the 2D 8x8 Hubbard model (n = 64, NQP = 8), same seeds and parameters.

Measurement is FP64 from the configuration in both paths, so a chain that meets no
Metropolis decision within the FP32 weight error of its threshold holds exactly the FP64
path's configurations; the refresh drift |ln|IP|_refreshed - ln|IP|_tracked| measures that
weight error directly.
"""
import numpy as np
import pytest

from mvmc_lib import lattice, mvmc

pytestmark = pytest.mark.gpu


def square8_inputs(tmp_path, interval=8, **over):
    lat = lattice()
    cfg = dict(lat.CONFIGS["square8"])
    cfg["interval"] = interval
    cfg.update(over)
    nl, init, dims = lat.write_inputs(str(tmp_path / "in"), **cfg)
    return nl, init, dims


def run(nl, init, precision, walkers, refresh, guard=0.0):
    eng = mvmc().Engine(nl, init, walkers=walkers, precision=precision, seed=99, refresh_sweeps=refresh,
                        refresh_guard=guard)
    eng.sample()
    e, ho, oo = eng.measure()
    out = dict(e=e, idx=eng.samples()["ele_idx"].reshape(walkers, -1), el=eng.local_energies(),
               o=eng.o_store(), stats=eng.refresh_stats())
    eng.close()
    return out


GUARD = 0.03  # the mixed path's refresh guard in these tests


NO_PROJECTION = dict(nmp=1, shifts=[(0, 0)], nsp_gauss_leg=1)


@pytest.fixture(scope="module")
def pair(tmp_path_factory):
    """One QP plane (no translation or spin projection), the case the FP32 inverse holds."""
    nl, init, dims = square8_inputs(tmp_path_factory.mktemp("sq8"), **NO_PROJECTION)
    W = 64
    return dims, run(nl, init, 64, W, 0), run(nl, init, 32, W, 8, GUARD)


def test_fp64_path_drift_without_projection_is_rounding_level(tmp_path):
    """One QP plane: the FP64 rank-2 updates stay at rounding level between C refreshes."""
    nl, init, _ = square8_inputs(tmp_path, interval=4, nmp=1, shifts=[(0, 0)], nsp_gauss_leg=1)
    assert run(nl, init, 64, 64, 0)["stats"]["drift_max"] <= 1e-9


def test_refresh_guard_bounds_fp64_drift_with_projection(tmp_path):
    """With 8 QP planes an accepted move can take one plane close to singular while the
    projected amplitude stays large; the reference's schedule then carries the amplified
    error to the next refresh. The guard recomputes right after such a move."""
    nl, init, _ = square8_inputs(tmp_path, interval=4)
    plain = run(nl, init, 64, 64, 0)["stats"]
    guarded = run(nl, init, 64, 64, 0, 1e-3)["stats"]
    assert guarded["guard_refreshes"] > 0
    assert guarded["drift_max"] <= 1e-6
    assert guarded["drift_max"] <= plain["drift_max"]


def test_mixed_path_drift_bounded_and_chains_match_fp64(pair):
    dims, f64, f32 = pair
    assert 0.0 < f32["stats"]["drift_max"] <= 5e-2
    same = np.all(f64["idx"] == f32["idx"], axis=1)
    assert same.mean() >= 0.5
    # identical configurations → identical FP64 measurement up to reduction order
    el64, el32 = f64["el"][same], f32["el"][same]
    assert np.all(np.abs(el64 - el32) <= 1e-10 * np.abs(el64).max())
    o64, o32 = f64["o"][same], f32["o"][same]
    assert np.all(np.abs(o64 - o32) <= 1e-10 * (1.0 + np.abs(o64).max()))


def test_mixed_path_energy_within_statistics_of_fp64(pair):
    dims, f64, f32 = pair
    err = np.std(f64["el"]) / np.sqrt(len(f64["el"]))
    assert abs(f32["e"][1] - f64["e"][1]) <= 5 * err + 1e-9


def test_guard_reduces_mixed_drift_with_projection(tmp_path):
    """Eight QP planes: FP32 inverses lose the amplitude between refreshes (the rounding
    of the stored inverse enters every ratio with the condition number of the plane);
    the guard's extra refreshes cut the loss by orders of magnitude but do not bring it
    to rounding level."""
    nl, init, _ = square8_inputs(tmp_path, interval=4)
    plain = run(nl, init, 32, 32, 2, 0.0)["stats"]
    guarded = run(nl, init, 32, 32, 2, 0.1)["stats"]
    assert guarded["guard_refreshes"] > 0
    assert guarded["drift_max"] * 10 <= plain["drift_max"]


def sr_update(nl, init, sr_precision, walkers=1024, sr_gram=0):
    eng = mvmc().Engine(nl, init, walkers=walkers, precision=64, seed=7, sr_precision=sr_precision,
                        sr_gram=sr_gram)
    p0 = eng.parameters()
    eng.sample()
    eng.measure()
    rc, info = eng.sr_cg()
    dp = eng.parameters() - p0
    eng.close()
    return rc, info, dp


@pytest.mark.parametrize("sr_precision,sr_gram,bound", [(32, 0, 1e-2), (16, 0, 5e-2), (32, 1, 1e-2), (16, 1, 5e-2)])
def test_reduced_precision_sr_operator_update_error(tmp_path, sr_precision, sr_gram, bound):
    """The SR parameter update with the FP32 / BF16 centred, column-scaled sample matrix
    (one pass per CG product) and with its Gram formed on the tensor cores (TF32 / BF16
    inputs, FP32 accumulation) against the FP64 operator on identical samples (same seeds,
    FP64 sampling)."""
    nl, init, _ = square8_inputs(tmp_path, interval=2)
    rc64, info64, d64 = sr_update(nl, init, 64)
    rc, info, d = sr_update(nl, init, sr_precision, sr_gram=sr_gram)
    assert rc == rc64 == 0
    assert np.array_equal(info[:4], info64[:4]), (info, info64)  # same active set
    assert np.linalg.norm(d64) > 0 and np.linalg.norm(d) > 0, (info, info64)
    err = np.linalg.norm(d - d64) / np.linalg.norm(d64)
    assert err <= bound, (err, info[8], info64[8])
