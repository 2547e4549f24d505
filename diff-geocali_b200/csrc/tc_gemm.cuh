// tc_gemm.cuh -- launch interface of the tcgen05 BF16 GEMM.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace dgc {

struct GemmArgs {
    const __nv_bfloat16* A;  // [M][lda], row-major (K contiguous)
    const __nv_bfloat16* B;  // [N][ldb], row-major (K contiguous)
    void* C;                 // [M][ldc], fp32 or bf16
    const float* bias;       // [N] or null
    int M, N, K, lda, ldb, ldc;
    int c_bf16;      // store bf16 (else fp32)
    int relu;        // max(x, 0) after the bias
    int accumulate;  // fp32 only: C += result
    float alpha;     // result = alpha * A B^T (+ bias)
    int* error;      // device word set to 1 when a pipeline wait times out
    int k_tiles_per_split;  // > 0: split K over gridDim.z CTAs, fp32 atomic epilogue
};

int tc_gemm(const GemmArgs& p, cudaStream_t s);

}  // namespace dgc
