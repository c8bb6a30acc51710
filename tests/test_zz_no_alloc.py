"""The allocation-free SR-CG entry point against the allocating one.

mvmc_b200_cg_solve_noalloc exists for callers that own all device memory through their
own allocator and cannot let the library call cudaMalloc. The test gives it device
buffers made by the caller (torch here), runs it twice in a row on the same buffers —
the second call starts from whatever the first left in the shared scratch array — and
checks both results against mvmc_b200_cg_solve (the entry point that allocates) on the
same operands: identical C status, solutions within 1e-12 relative. This file is
collected last so that a stop-at-first-failure run has already run every other test.
"""
import numpy as np
import pytest

from mvmc_lib import mvmc

pytestmark = pytest.mark.gpu


def operands(seed, ns, na):
    rng = np.random.default_rng(seed)
    smp = rng.normal(size=(ns, na))
    mean = smp.mean(axis=0)
    diag = (smp * smp).mean(axis=0) - mean * mean
    g = rng.normal(size=na)
    return smp, mean, diag, g


def test_noalloc_cg_matches_allocating_cg_on_two_calls():
    import torch

    m = mvmc()
    dev = torch.device("cuda:0")
    for seed, (ns, na), max_iter in ((3, (300, 40), 40), (4, (2048, 160), 60)):
        smp, mean, diag, g = operands(seed, ns, na)
        ref_status, ref_x = m.cg_solve(smp, mean, diag, g, 1.0 / ns, 0.02, 1e-10, max_iter)
        t = {k: torch.tensor(v, dtype=torch.float64, device=dev)
             for k, v in dict(smp=smp.ravel(), mean=mean, diag=diag, g=g).items()}
        for call in range(2):
            x = torch.full((na,), float("nan"), dtype=torch.float64, device=dev)
            res = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
            rc = m.cg_solve_noalloc(t["smp"].data_ptr(), ns, na, t["mean"].data_ptr(), t["diag"].data_ptr(),
                                    t["g"].data_ptr(), 1.0 / ns, 0.02, 1e-10, max_iter, False,
                                    x.data_ptr(), res.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            got = x.cpu().numpy()
            assert int(res[1].item()) == ref_status, (seed, call)
            assert np.all(np.abs(got - ref_x) <= 1e-12 * np.abs(ref_x).max()), (seed, call)


def test_noalloc_cg_rejects_problems_beyond_its_scratch_array():
    import torch

    m = mvmc()
    na, ns = 8, 1 << 21  # the row products alone need more than 2^20 doubles
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    with pytest.raises(RuntimeError, match="scratch"):
        m.cg_solve_noalloc(p, ns, na, p, p, p, 1.0, 0.0, 0.0, 1, False, p, p)
