"""The allocation-free FDK filter, dgc_fdk_filter_noalloc, through the C ABI.

Some callers cannot allocate device memory: an application that owns the GPU
and hands each library a fixed memory budget, a plugin that must not grow the
process's device footprint, or a latency-bound pipeline that keeps cudaMalloc
and cudaFree out of its steady state.  For them the filter keeps its only
scratch (the filter taps) in a static device array of at most
DGC_FDK_NOALLOC_MAX_U = 8192 floats, shared by all calls.

The filter's taps are computed on the device at every call, into a static
device array of 98 KiB shared by all calls (the spectrum in DGC_FDK_NOALLOC_MAX_U
+ 1 doubles, the taps in DGC_FDK_NOALLOC_MAX_U = 8192 floats).

The tests call the entry point several times in a row with different detector
widths (so taps left over from one call would show in the next) and check each
result against the workspace entry point dgc_fdk_filter, within the filter's
tolerance (rel-L2 1e-5); that repeated calls leave the device's free memory
and torch's allocation count unchanged; and that a width above the maximum is
refused.  This file sorts last so that a failing run has already
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
    from dgc_b200 import _native

    lib = _native.lib()
    rng = np.random.default_rng(5)
    cases = [((6, 384, 40), 0.9, 0.8), ((3, 48, 33), 1.0, 1.0), ((1, MAX_U, 8), 0.5, 0.7)]
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
    from dgc_b200 import _native

    lib = _native.lib()
    p = torch.zeros((1, 2, 2), device="cuda")
    rc = lib.dgc_fdk_filter_noalloc(p.data_ptr(), 1, MAX_U + 1, 2, 1.0, p.data_ptr(), p.data_ptr(),
                                    0.8, p.data_ptr(), None)
    assert rc == 4
    assert b"exceeds" in lib.dgc_last_error()


def test_noalloc_filter_allocates_nothing():
    from dgc_b200 import _native

    lib = _native.lib()
    rng = np.random.default_rng(9)
    shapes = [(4, 256, 24), (2, 1000, 17), (4, 256, 24), (1, MAX_U, 4)]
    inputs = []
    for A, U, V in shapes:
        p = torch.tensor(rng.random((A, U, V)), dtype=torch.float32, device="cuda")
        sod = torch.full((A,), 600.0, device="cuda")
        sid = torch.full((A,), 1000.0, device="cuda")
        inputs.append((p, sod, sid, torch.empty_like(p)))
    stream = torch.cuda.current_stream().cuda_stream

    def call(p, sod, sid, out):
        A, U, V = p.shape
        rc = lib.dgc_fdk_filter_noalloc(p.data_ptr(), A, U, V, 1.0, sod.data_ptr(), sid.data_ptr(),
                                        0.8, out.data_ptr(), stream)
        assert rc == 0, lib.dgc_last_error()

    call(*inputs[0])  # warm-up: loads the kernels on this device
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    allocated_before = torch.cuda.memory_allocated()
    for _ in range(3):
        for args in inputs:
            call(*args)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert torch.cuda.memory_allocated() == allocated_before
