// tma.cuh -- tensor-memory-accelerator plumbing shared by the kernels that
// stage tiles with cp.async.bulk.tensor (this GPU's memory only; no cluster
// multicast anywhere in this library).
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace dgc {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); null if the driver does not provide it.
EncodeTiledFn encode_tiled();

// Iterations of a bounded mbarrier wait before it gives up (far above any
// completion time of a legitimate copy).
constexpr long long kTmaWaitLimit = 1LL << 24;

__device__ __forceinline__ uint32_t tma_smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tma_mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void tma_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void tma_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// Bounded wait for the phase of the given parity; false on timeout.
__device__ __forceinline__ bool tma_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kTmaWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 3-D tiled load into shared memory, completing on mbarrier `bar`.  The
// innermost coordinate x times the element size must be a multiple of 16
// bytes (the caller's coordinates guarantee it); other coordinates may be
// negative or beyond the tensor (zero fill).
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

}  // namespace dgc
