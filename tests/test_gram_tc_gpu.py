"""Gram matrix of the SR samples on the tensor cores (tcgen05.mma, BF16 or TF32 inputs, FP32
accumulation) against an FP64 Gram of the same rounded inputs."""
import numpy as np
import pytest

from mvmc_lib import mvmc

pytestmark = pytest.mark.gpu


def to_bf16(x):
    """FP64 → FP32 (round to nearest) → BF16 (round to nearest even), as FP64 values."""
    f = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (f + 0x7FFF + ((f >> 16) & 1)) >> 16 << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def to_tf32(x, mode):
    f = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    if mode == "trunc":
        r = f & ~np.uint64(0x1FFF)
    else:
        r = (f + 0xFFF + ((f >> 13) & 1)) >> 13 << 13
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("ns,na", [(1000, 300), (4100, 257), (64, 128)])
def test_bf16_gram_matches_fp64_gram_of_rounded_inputs(ns, na):
    """Padding in both dimensions (samples to 64, parameters to 128), several output tiles
    (diagonal and mirrored off-diagonal) and several K slabs through the 4-stage ring:
    every entry within 1e-4·Σ|x_i||x_j| of the FP64 Gram of the BF16-rounded samples (FP32
    accumulation), and G exactly symmetric."""
    rng = np.random.default_rng(ns + na)
    x = rng.normal(size=(ns, na)) * rng.uniform(0.1, 3.0, size=na)
    g = mvmc().gram_tc(x, 16)
    xb = to_bf16(x)
    ref = xb.T @ xb
    bound = 1e-4 * (np.abs(xb).T @ np.abs(xb))
    assert np.all(np.abs(g - ref) <= bound), np.max(np.abs(g - ref) / bound)
    assert np.array_equal(g, g.T)


@pytest.mark.parametrize("ns,na", [(1000, 300), (2048, 129)])
def test_tf32_gram_matches_fp64_gram_of_tf32_inputs(ns, na):
    """TF32 inputs (FP32 samples read with a 10-bit mantissa): every entry within
    1e-4·Σ|x_i||x_j| of the FP64 Gram of the samples reduced to TF32."""
    rng = np.random.default_rng(7 + ns)
    x = rng.normal(size=(ns, na))
    g = mvmc().gram_tc(x, 32)
    errs = []
    for mode in ("trunc", "rn"):
        xt = to_tf32(x, mode)
        ref = xt.T @ xt
        bound = 1e-4 * (np.abs(xt).T @ np.abs(xt))
        errs.append(np.max(np.abs(g - ref) / bound))
    assert min(errs) <= 1.0, errs
    assert np.array_equal(g, g.T)


@pytest.mark.parametrize("precision", [16, 32])
def test_gram_at_the_sr_configuration_shape(precision):
    """The 2D 16x16 SR configuration's shape (8192 samples × 4226 active parameters): 400
    random entries against FP64 dot products of the rounded samples (1e-4 relative to
    Σ|x_i||x_j|), the matrix exactly symmetric."""
    rng = np.random.default_rng(precision)
    x = rng.normal(size=(8192, 4226))
    g = mvmc().gram_tc(x, precision)
    xr = to_bf16(x) if precision == 16 else None
    i = rng.integers(0, 4226, 400)
    j = rng.integers(0, 4226, 400)
    for a, b in zip(i, j):
        if precision == 16:
            ref, scale = xr[:, a] @ xr[:, b], np.abs(xr[:, a]) @ np.abs(xr[:, b])
        else:
            cand = [to_tf32(x[:, [a, b]], m) for m in ("trunc", "rn")]
            ref = min((c[:, 0] @ c[:, 1] for c in cand), key=lambda r: abs(r - g[a, b]))
            scale = np.abs(x[:, a]) @ np.abs(x[:, b])
        assert abs(g[a, b] - ref) <= 1e-4 * scale, (a, b, g[a, b], ref)
    assert np.array_equal(g, g.T)
