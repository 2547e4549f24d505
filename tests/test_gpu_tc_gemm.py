"""The tcgen05 BF16 GEMM (dgc_gemm_bf16) against an FP32 matmul of the same
bf16 inputs: ragged M/N/K, all three tile widths, bias + ReLU, bf16 output,
accumulation into fp32, split-K; the TMA pipeline (default) and the cp.async
pipeline (DGC_GEMM=cpasync)."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def run(A, B, C, bias=None, relu=False, accumulate=False, alpha=1.0):
    from dgc_b200 import _native

    lib = _native.lib()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    M, K = A.shape
    N = B.shape[0]
    rc = lib.dgc_gemm_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(),
                           None if bias is None else bias.data_ptr(), M, N, K, A.stride(0),
                           B.stride(0), C.stride(0), int(C.dtype == torch.bfloat16), int(relu),
                           int(accumulate), float(alpha), err.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.dgc_last_error()
    torch.cuda.synchronize()
    assert err.item() == 0
    return C


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 64, 16), (300, 200, 72), (1000, 64, 256),
                                   (2048, 256, 2304), (7, 24, 8), (513, 136, 136),
                                   (64, 200, 8192), (32, 96, 4104), (18944, 264, 72),
                                   (9000, 520, 136), (9400, 1000, 200)])
@pytest.mark.parametrize("pipeline", ["tma", "cpasync"])
def test_gemm_matches_fp32(M, N, K, pipeline, monkeypatch):
    """(64, 200, 8192) and (32, 96, 4104) take the split-K path (few output
    tiles, long K); (9000, 520, 136) the 128 x 256 tiles; (18944, 264, 72)
    and (9400, 1000, 200) the 256 x 256 tiles of two accumulators."""
    if pipeline == "cpasync":
        monkeypatch.setenv("DGC_GEMM", "cpasync")
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    want = A.float() @ B.float().t()
    C = torch.full((M, N), float("nan"), device="cuda")
    from dgc_b200 import _native

    with _native.trace() as tr:
        got = run(A, B, C)
    want_kernel = "tc_gemm_tma_kernel" if pipeline == "tma" else "tc_gemm_kernel"
    assert {n for n, _ in tr.records} == {want_kernel}
    scale = (A.float().abs() @ B.float().abs().t()).clamp_min(1.0)
    assert ((got - want).abs() / scale).max().item() < 1e-5


def test_gemm_epilogues():
    g = torch.Generator(device="cuda").manual_seed(3)
    M, N, K = 260, 96, 40
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    ref = A.float() @ B.float().t()
    out = run(A, B, torch.empty(M, N, device="cuda", dtype=torch.bfloat16), bias=bias, relu=True)
    torch.testing.assert_close(out.float(), torch.relu(ref + bias), rtol=1e-2, atol=1e-2)
    acc = torch.randn(M, N, device="cuda", generator=g)
    want = acc + 0.5 * ref
    run(A, B, acc, accumulate=True, alpha=0.5)
    torch.testing.assert_close(acc, want, rtol=1e-5, atol=1e-4)
    # strided operands (row stride larger than K)
    Aw = torch.randn(M, 64, device="cuda", generator=g).to(torch.bfloat16)[:, :K]
    Bw = torch.randn(N, 48, device="cuda", generator=g).to(torch.bfloat16)[:, :K]
    out2 = run(Aw, Bw, torch.empty(M, N, device="cuda"))
    torch.testing.assert_close(out2, Aw.float() @ Bw.float().t(), rtol=1e-5, atol=1e-4)


def test_split_k_into_column_slice():
    """Split-K zeroes and sums only the M x N window of a strided C: the
    columns of the wider array around it keep their values."""
    g = torch.Generator(device="cuda").manual_seed(5)
    M, N, K = 48, 40, 6144
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    wide = torch.full((M, N + 24), 7.0, device="cuda")
    run(A, B, wide[:, 8:8 + N])
    want = A.float() @ B.float().t()
    scale = (A.float().abs() @ B.float().abs().t()).clamp_min(1.0)
    assert ((wide[:, 8:8 + N] - want).abs() / scale).max().item() < 1e-5
    assert torch.all(wide[:, :8] == 7.0) and torch.all(wide[:, 8 + N:] == 7.0)
    # accumulate=True adds the split partial sums to what C holds
    acc = wide[:, 8:8 + N].clone()
    run(A, B, acc, accumulate=True, alpha=-1.0)
    assert (acc.abs() / scale).max().item() < 1e-5
