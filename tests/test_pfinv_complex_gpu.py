"""Complex skew Pfaffian + inverse on the device (mvmc_b200_pfinv_batch_complex): the
reference's complex test matrices (tests/fixtures/pfapack/complex_n*, whose goldens were
removed upstream, so parity is by identity as in crates/pfapack/tests/
fixed_matrix_identities.rs: Pf² = det, inverse residual), seeded batches against a
Parlett–Reid Pfaffian in numpy, the real entry point on real-valued planes, and a
singular plane."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from mvmc_lib import mvmc

pytestmark = pytest.mark.gpu
D = os.path.join(ol.GOLDEN, "pfapack_complex")


def read_complex(path):
    vals = []
    for line in open(path):
        t = line.split()
        if len(t) != 2 or line.startswith("#"):
            continue
        try:
            vals.append(float(t[0]) + 1j * float(t[1]))
        except ValueError:  # the "kind", "n", "seed" header lines
            continue
    n = int(round(len(vals) ** 0.5))
    return np.array(vals).reshape(n, n), n


def pfaffian_parlett_reid(a):
    """Pf of a skew matrix by Parlett–Reid with row/column pivoting (textbook form)."""
    a = np.array(a, dtype=np.complex128)
    n = a.shape[0]
    pf = 1.0 + 0.0j
    for k in range(0, n - 1, 2):
        kp = k + 1 + int(np.abs(a[k, k + 1:]).argmax())
        if kp != k + 1:
            a[[k + 1, kp], :] = a[[kp, k + 1], :]
            a[:, [k + 1, kp]] = a[:, [kp, k + 1]]
            pf = -pf
        if a[k, k + 1] == 0:
            return 0.0
        pf *= a[k, k + 1]
        if k + 2 < n:
            tau = a[k, k + 2:] / a[k, k + 1]
            a[k + 2:, k + 2:] += np.outer(tau, a[k + 2:, k + 1]) - np.outer(a[k + 2:, k + 1], tau)
    return pf


def skew_complex(rng, n, planes):
    u = np.triu(rng.normal(size=(planes, n, n)) + 1j * rng.normal(size=(planes, n, n)), 1)
    x = u - np.transpose(u, (0, 2, 1))
    i = np.arange(0, n, 2)
    x[:, i, i + 1] += 0.5
    x[:, i + 1, i] -= 0.5
    return x


def colmajor(x):
    return np.ascontiguousarray(np.transpose(x, (0, 2, 1))).ravel()


@pytest.mark.parametrize("name", sorted(os.listdir(D)))
def test_reference_complex_matrices_satisfy_the_identities(name):
    x, n = read_complex(os.path.join(D, name))
    assert np.allclose(x, -x.T)
    pf, inv, st = mvmc().pfinv_batch_complex(colmajor(x[None]), n, 1)
    assert st[0] == 0
    xi = inv.reshape(n, n).T
    det = np.linalg.det(x)
    assert abs(pf[0] ** 2 - det) <= n * 1e-12 * abs(det)
    resid = np.abs(xi @ x - np.eye(n)).max() / (np.abs(x).max() * np.abs(xi).max())
    assert resid <= 64 * np.finfo(float).eps * n


@pytest.mark.parametrize("n,planes", [(2, 5), (6, 33), (16, 64), (64, 20), (96, 4)])
def test_seeded_batches_match_parlett_reid(n, planes):
    x = skew_complex(np.random.default_rng(n), n, planes)
    pf, inv, st = mvmc().pfinv_batch_complex(colmajor(x), n, planes)
    assert (st == 0).all()
    inv = inv.reshape(planes, n, n)
    for p in range(planes):
        ref = pfaffian_parlett_reid(x[p])
        assert abs(pf[p] - ref) <= 1e-11 * n * abs(ref), (p, pf[p], ref)
        xi = inv[p].T
        assert np.abs(xi @ x[p] - np.eye(n)).max() <= 1e-11 * n


def test_real_valued_planes_match_the_real_entry_point():
    rng = np.random.default_rng(4)
    n, planes = 32, 16
    u = np.triu(rng.normal(size=(planes, n, n)), 1)
    x = u - np.transpose(u, (0, 2, 1))
    pf_c, inv_c, st_c = mvmc().pfinv_batch_complex(colmajor(x.astype(np.complex128)), n, planes)
    pf_r, inv_r, st_r = mvmc().pfinv_batch(colmajor(x), n, planes)
    assert (st_c == 0).all() and (st_r == 0).all()
    assert np.allclose(pf_c.real, pf_r, rtol=1e-12) and np.all(pf_c.imag == 0)
    assert np.allclose(inv_c.real, inv_r, rtol=1e-11, atol=1e-12 * np.abs(inv_r).max())


def test_singular_complex_plane_reports_its_pivot_row():
    x = np.zeros((1, 4, 4), dtype=np.complex128)
    x[0, 0, 1], x[0, 1, 0] = 1 + 1j, -1 - 1j
    pf, inv, st = mvmc().pfinv_batch_complex(colmajor(x), 4, 1)
    assert st[0] == 3 and pf[0] == 0


@pytest.mark.parametrize("scale", [1e-160, 1e160])
def test_tiny_and_huge_planes_factor_like_the_reference(scale):
    """Pivots are chosen by |Re| + |Im| (zsktf2's IZAMAX 1-norm) and the update coefficients
    are scaled by 1/a before they meet another entry, so planes whose entries lie below
    1e-154 or above 1e154 (where |z|² and products of two entries under- or overflow) still
    factor: the inverse is the unscaled one times 1/scale. For n = 2 the Pfaffian is scale
    times the unscaled one; for n = 8 it is scale⁴ (1e-640 underflows to 0 with status 0,
    1e640 overflows: status -1, the reference's non-finite Pfaffian)."""
    for n in (2, 8):
        x = skew_complex(np.random.default_rng(11 + n), n, 3)
        pf0, inv0, st0 = mvmc().pfinv_batch_complex(colmajor(x), n, 3)
        pf, inv, st = mvmc().pfinv_batch_complex(colmajor(x * scale), n, 3)
        assert (st0 == 0).all()
        want = -1 if (n == 8 and scale > 1) else 0
        assert (st == want).all(), st
        assert np.allclose(inv * scale, inv0, rtol=1e-12, atol=1e-12 * np.abs(inv0).max())
        if n == 2:
            assert np.allclose(pf, pf0 * scale, rtol=1e-14)


def test_device_buffer_entry_matches_the_host_entry():
    """mvmc_b200_pfinv_batch_complex_device on device buffers (torch allocations, the
    caller's stream) gives the host-buffer entry point's bits."""
    import ctypes
    import torch
    m = mvmc()
    n, planes = 24, 40
    x = colmajor(skew_complex(np.random.default_rng(5), n, planes))
    pf_h, inv_h, st_h = m.pfinv_batch_complex(x, n, planes)
    dx = torch.from_numpy(x.view(np.float64).copy()).cuda()
    dinv = torch.empty_like(dx)
    dpf = torch.zeros(2 * planes, dtype=torch.float64, device="cuda")
    dst = torch.zeros(planes, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = m.lib().mvmc_b200_pfinv_batch_complex_device(P(dx), n, planes, P(dpf), P(dinv), P(dst),
                                                      ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(dpf.cpu().numpy().view(np.complex128), pf_h)
    assert np.array_equal(dinv.cpu().numpy().view(np.complex128), inv_h)
    assert np.array_equal(dst.cpu().numpy(), st_h)


def test_batch_spanning_several_pipeline_chunks():
    """480 planes of n = 96 (71 MB, three ~32 MB chunks on the two-stream pipe): every
    inverse residual at rounding level and Pf² = det on every plane."""
    n, planes = 96, 480
    x = skew_complex(np.random.default_rng(17), n, planes)
    pf, inv, st = mvmc().pfinv_batch_complex(colmajor(x), n, planes)
    assert (st == 0).all()
    xi = np.transpose(inv.reshape(planes, n, n), (0, 2, 1))
    resid = np.abs(xi @ x - np.eye(n)).max(axis=(1, 2))
    assert resid.max() <= 1e-11 * n
    sign, logdet = np.linalg.slogdet(x)
    lpf2 = 2 * np.log(pf)
    assert np.allclose(np.exp(lpf2 - logdet), sign, rtol=1e-10 * n)
