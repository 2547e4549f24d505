"""The allocation-free FDK filter, dgc_fdk_filter_noalloc, through the C ABI.

Some callers cannot allocate device memory: an application that owns the GPU
and hands each library a fixed memory budget, a plugin that must not grow the
process's device footprint, or a latency-bound pipeline that keeps cudaMalloc
and cudaFree out of its steady state.  For them the filter keeps its only
scratch (the filter taps) in a static device array of at most
DGC_FDK_NOALLOC_MAX_U = 8192 floats, shared by all calls.

The test calls the entry point twice in a row with different detector widths
(so taps left over from the first call would show in the second) and checks
each result against the workspace entry point dgc_fdk_filter, within the
filter's tolerance (rel-L2 1e-5); it also checks that a width above the
maximum is refused.  This file sorts last so that a failing run has already
run every other test; it also passes on its own in a fresh process.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_U = 8192


def rel_l2(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


def with_workspace(lib, p, px, sod, sid, alpha):
    A, U, V = p.shape
    out = torch.empty_like(p)
    n = lib.dgc_fdk_filter_workspace_bytes(A, U, V)
    ws = torch.empty(n, dtype=torch.uint8, device=p.device)
    rc = lib.dgc_fdk_filter(p.data_ptr(), A, U, V, px, sod.data_ptr(), sid.data_ptr(), alpha,
                            out.data_ptr(), ws.data_ptr(), n, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.dgc_last_error()
    return out


def without_allocation(lib, p, px, sod, sid, alpha):
    A, U, V = p.shape
    out = torch.full_like(p, float("nan"))
    rc = lib.dgc_fdk_filter_noalloc(p.data_ptr(), A, U, V, px, sod.data_ptr(), sid.data_ptr(),
                                    alpha, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.dgc_last_error()
    return out


def test_noalloc_filter_matches_workspace_filter():
    from cbct_backprojector import _native

    lib = _native.lib()
    rng = np.random.default_rng(5)
    cases = [((6, 384, 40), 0.9, 0.8), ((3, 48, 33), 1.0, 1.0)]
    for (A, U, V), px, alpha in cases:
        p = torch.tensor(rng.random((A, U, V)) * 3, dtype=torch.float32, device="cuda")
        sod = torch.tensor(600 + rng.normal(0, 5, A), dtype=torch.float32, device="cuda")
        sid = torch.tensor(1000 + rng.normal(0, 5, A), dtype=torch.float32, device="cuda")
        got = without_allocation(lib, p, px, sod, sid, alpha)
        want = with_workspace(lib, p, px, sod, sid, alpha)
        torch.cuda.synchronize()
        assert torch.isfinite(got).all()
        assert rel_l2(got, want) < 1e-5


def test_noalloc_filter_rejects_oversized_detector():
    from cbct_backprojector import _native

    lib = _native.lib()
    p = torch.zeros((1, 2, 2), device="cuda")
    rc = lib.dgc_fdk_filter_noalloc(p.data_ptr(), 1, MAX_U + 1, 2, 1.0, p.data_ptr(), p.data_ptr(),
                                    0.8, p.data_ptr(), None)
    assert rc == 4
    assert b"exceeds" in lib.dgc_last_error()
