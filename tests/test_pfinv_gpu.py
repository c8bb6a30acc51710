"""K1 parity: batched Pfaffian + inverse on the GPU against the oracle (pfapack order)."""
import os

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def mvmc():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mvmc_b200", os.path.join(ol.ROOT, "mvmc-rs_b200", "mvmc_b200.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def skew_batch(rng, n, planes):
    """A_ij ~ N(0,1), i<j, plus 0.5·J padding (block-diagonal [[0,1],[-1,0]])."""
    u = np.triu(rng.normal(size=(planes, n, n)), 1)
    x = u - np.transpose(u, (0, 2, 1))
    for i in range(0, n, 2):
        x[:, i, i + 1] += 0.5
        x[:, i + 1, i] -= 0.5
    return x


def colmajor(x):
    return np.ascontiguousarray(np.transpose(x, (0, 2, 1))).ravel()


@pytest.mark.parametrize("n,planes", [(2, 7), (4, 33), (16, 64), (64, 128), (128, 16), (224, 4)])
def test_pfinv_matches_oracle(n, planes):
    m = mvmc()
    x = skew_batch(np.random.default_rng(n), n, planes)
    xc = colmajor(x)
    pf, inv, st = m.pfinv_batch(xc, n, planes)
    opf, oinv, ost = ol.pfinv_batch(xc, n, planes)
    assert (st == 0).all() and (ost == 0).all()
    # ln|Pf| and sign within 1e-12 relative of pfapack; inverse within 1e-12 of its norm
    assert np.all(np.sign(pf) == np.sign(opf))
    assert np.max(np.abs(pf - opf) / np.abs(opf)) < 1e-12 * max(1, n / 16)
    inv = inv.reshape(planes, n, n)
    oinv = oinv.reshape(planes, n, n)
    scale = np.abs(oinv).max(axis=(1, 2), keepdims=True)
    assert np.max(np.abs(inv - oinv) / scale) < 1e-12 * max(1, n / 16)


def test_pfinv_mixed_sizes_one_launch():
    m = mvmc()
    rng = np.random.default_rng(7)
    sizes = [32, 48, 64, 96, 128] * 4
    xs = [skew_batch(rng, n, 1) for n in sizes]
    x = np.concatenate([colmajor(a) for a in xs])
    pf, inv, st = m.pfinv_batch_mixed(x, sizes, 64)
    off = 0
    for k, n in enumerate(sizes):
        opf, oinv, ost = ol.pfinv_batch(x[off:off + n * n], n, 1)
        assert st[k] == 0
        assert abs(pf[k] - opf[0]) / abs(opf[0]) < 1e-12 * max(1, n / 16)
        d = np.abs(inv[off:off + n * n] - oinv).max() / np.abs(oinv).max()
        assert d < 1e-12 * max(1, n / 16)
        off += n * n


def test_pfinv_fp32_variant_error_is_bounded():
    m = mvmc()
    rng = np.random.default_rng(11)
    n, planes = 64, 32
    x = colmajor(skew_batch(rng, n, planes))
    pf, inv, st = m.pfinv_batch_mixed(x, [n] * planes, 32)
    opf, oinv, _ = ol.pfinv_batch(x, n, planes)
    assert (st == 0).all()
    assert np.max(np.abs(pf - opf) / np.abs(opf)) < 1e-3
    assert np.max(np.abs(inv - oinv)) / np.abs(oinv).max() < 1e-3


def test_pfinv_reference_fixture_matrices():
    m = mvmc()
    d = os.path.join(ol.GOLDEN, "pfapack")
    for name in sorted(os.listdir(d)):
        vals = [float(l) for l in open(os.path.join(d, name)) if l.strip() and not l.startswith("#") and " " not in l.strip()]
        n = int(round(len(vals) ** 0.5))
        x = np.array(vals).reshape(n, n)
        pf, inv, st = m.pfinv_batch(x.T.ravel(), n, 1)
        assert st[0] == 0
        xi = inv.reshape(n, n).T
        assert abs(2 * np.log(abs(pf[0])) - np.linalg.slogdet(x)[1]) <= n * 1e-13
        resid = np.abs(xi @ x - np.eye(n)).max() / (np.abs(x).max() * np.abs(xi).max())
        assert resid <= 64 * np.finfo(float).eps * n


def test_pfinv_singular_plane_reports_status():
    m = mvmc()
    x = np.zeros((2, 4, 4))
    x[0, 0, 1], x[0, 1, 0] = 1.0, -1.0  # rank 2
    x[1] = skew_batch(np.random.default_rng(3), 4, 1)[0]
    pf, inv, st = m.pfinv_batch(colmajor(x), 4, 2)
    assert st[0] > 0 and pf[0] == 0.0
    assert st[1] == 0


@pytest.mark.parametrize("n,tiles", [(32, ["16x2", "8x4"]), (64, ["16x4", "8x8"]), (96, ["32x4", "16x8"]),
                                     (128, ["32x4", "16x8"])])
@pytest.mark.parametrize("precision", [64, 32])
def test_autotuner_candidates_give_identical_bits(n, tiles, precision, monkeypatch):
    """The tile shapes the autotuner chooses between compute every element with the same
    operations: Pf, the inverse and the status agree bitwise with the tuned default."""
    m = mvmc()
    x = colmajor(skew_batch(np.random.default_rng(3 * n), n, 300))
    base = m.pfinv_batch_mixed(x, [n] * 300, precision)
    for t in tiles:
        monkeypatch.setenv("MVMC_B200_PFINV_TILE", t)
        got = m.pfinv_batch_mixed(x, [n] * 300, precision)
        for a, b in zip(base, got):
            assert np.array_equal(a, b), t
    monkeypatch.setenv("MVMC_B200_PFINV_TILE", "")


def device_uniform(xc, n, planes, precision):
    """mvmc_b200_pfinv_batch_device on a uniform batch (sizes NULL) in device buffers."""
    import ctypes
    import torch
    x = torch.from_numpy(np.ascontiguousarray(xc)).cuda()
    inv = torch.empty_like(x)
    pf = torch.zeros(planes, dtype=torch.float64, device="cuda")
    st = torch.zeros(planes, dtype=torch.int32, device="cuda")
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = mvmc().lib().mvmc_b200_pfinv_batch_device(P(x), None, None, n, planes, n, P(pf), P(inv), P(st), precision,
                                                   None)
    assert rc >= 0
    torch.cuda.synchronize()
    return pf.cpu().numpy(), inv.cpu().numpy(), st.cpu().numpy()


@pytest.mark.parametrize("n", [32, 64])
def test_uniform_batch_kernel_matches_oracle_and_flags_singular_planes(n):
    """Uniform batches of side 32 and 64 run the one-barrier register sweep: Pf and X⁻¹
    within the oracle bounds in FP64, within 1e-3 in FP32; a rank-deficient plane in the
    batch (rank 2, and a plane with one zero row and column) reports its status and Pf 0
    without disturbing its neighbours; the result equals the two-barrier tiles' within
    rounding."""
    m = mvmc()
    planes = 300
    x = skew_batch(np.random.default_rng(100 + n), n, planes)
    x[7] = 0.0
    x[7, 0, 1], x[7, 1, 0] = 1.0, -1.0
    x[11, 5, :] = 0.0
    x[11, :, 5] = 0.0
    xc = colmajor(x)
    ok = np.ones(planes, bool)
    ok[[7, 11]] = False
    pf, inv, st = m.pfinv_batch(xc, n, planes)
    opf, oinv, ost = ol.pfinv_batch(xc, n, planes)
    assert st[7] > 0 and st[11] > 0 and pf[7] == 0.0 and pf[11] == 0.0
    assert (st[ok] == 0).all() and (ost[ok] == 0).all()
    assert np.all(np.sign(pf[ok]) == np.sign(opf[ok]))
    assert np.max(np.abs(pf[ok] - opf[ok]) / np.abs(opf[ok])) < 1e-12 * max(1, n / 16)
    inv = inv.reshape(planes, n, n)[ok]
    oinv = oinv.reshape(planes, n, n)[ok]
    scale = np.abs(oinv).max(axis=(1, 2), keepdims=True)
    assert np.max(np.abs(inv - oinv) / scale) < 1e-12 * max(1, n / 16)
    pf32, inv32, st32 = device_uniform(xc, n, planes, 32)
    assert (st32[ok] == 0).all() and st32[7] > 0 and st32[11] > 0
    assert np.max(np.abs(pf32[ok] - opf[ok]) / np.abs(opf[ok])) < 1e-3
    assert np.max(np.abs(inv32.reshape(planes, n, n)[ok] - oinv) / scale) < 1e-3
