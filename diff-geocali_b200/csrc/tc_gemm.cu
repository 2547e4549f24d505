// tc_gemm.cu -- BF16 x BF16 -> FP32 GEMM on the sm_100 5th-generation tensor
// cores (tcgen05.mma, accumulators in tensor memory), for the convolution
// layers of the warm-start network.  No counterpart in the reference.
//
//   C[m, n] (+)= sum_k A[m, k] * B[n, k]  (+ bias[n], optional ReLU)
//
// A (M x K) and B (N x K) are row-major bf16 ("K-major"); C is fp32 or bf16.
//
// Structure of a CTA (128 threads, one 128 x BN output tile):
//   * warp 0 allocates BN tensor-memory columns (a 128-lane x BN fp32
//     accumulator) and frees them at the end;
//   * all threads stage 128 x 64 tiles of A and BN x 64 tiles of B into shared
//     memory with cp.async, four stages deep, in the 128-byte-swizzled K-major
//     layout: row r of a tile is 128 contiguous bytes (its 64 K elements) at
//     r*128, its 16-byte chunk j stored at chunk j ^ (r % 8); eight
//     consecutive threads copy one row, so the global reads are 128-byte
//     coalesced and the shared-memory writes conflict-free (SBO = 1024 B
//     between 8-row groups; the K = 16 step of an MMA advances the start
//     address by 32 B inside the swizzle atom);
//   * one elected thread issues four tcgen05.mma (M=128, N=BN, K=16) per stage
//     and commits them to the stage's mbarrier, which releases the stage for
//     the next prefetch and, after the last stage, signals the epilogue;
//   * the four warps read their 32 accumulator lanes with tcgen05.ld, apply
//     bias / ReLU / accumulate and store.
// Every mbarrier wait is bounded; a timeout sets the error word, skips the
// epilogue and still frees the tensor memory.
#include <cuda.h>

#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tma.cuh"

namespace dgc {

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<EncodeTiledFn>(nullptr);
        return reinterpret_cast<EncodeTiledFn>(ptr);
    }();
    return fn;
}

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kStages = 4;
constexpr long long kWaitLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; ++i) {
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

// Shared-memory matrix descriptor, K-major, 128-byte swizzle (sm_100 format:
// start >> 4 in [0,14), LBO >> 4 in [16,30) (16 B, unused by swizzled
// K-major), SBO >> 4 in [32,46) (1024 B between 8-row groups), version 1 at
// bit 46, base offset 0 (atoms 1024-byte aligned), layout type 2 =
// SWIZZLE_128B in [61,64)).
__device__ __forceinline__ uint64_t kmajor_sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(16u >> 4) << 16;
    d |= static_cast<uint64_t>(1024u >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}

// Instruction descriptor of kind::f16 with bf16 A and B, fp32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage one K-slice: 'rows' x 64 bf16 of a K-major matrix into the 128-byte
// swizzled layout (16-byte chunk j of row r at r*128 + ((j ^ (r & 7)) * 16)).
// Out-of-range rows or K chunks are zero-filled.
template <int ROWS>
__device__ __forceinline__ void stage_tile(uint32_t sbase, const __nv_bfloat16* g, int ld,
                                           int row0, int nrows, int k0, int K) {
    constexpr int kChunks = ROWS * (kBK / 8);
#pragma unroll 4
    for (int c = threadIdx.x; c < kChunks; c += 128) {
        const int r = c >> 3, j = c & 7;
        const int row = row0 + r, k = k0 + j * 8;
        const bool ok = row < nrows && k < K;
        const __nv_bfloat16* src = ok ? g + (long long)row * ld + k : g;
        cp_async16(sbase + static_cast<uint32_t>(r * 128 + ((j ^ (r & 7)) << 4)), src, ok ? 16 : 0);
    }
}

// Epilogue: the four warps read their 32 accumulator lanes (rows) with
// tcgen05.ld, 16 columns at a time, and apply alpha / bias / ReLU /
// accumulate (or the split-K atomic sum) on the way to C.
template <int BN>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& p, uint32_t tmem, int m0, int n0,
                                              bool has_k, bool split) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_load16(lane_addr + c0, v);
            if (row < p.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col >= p.N) break;
                    float x = has_k ? v[j] : 0.0f;
                    x *= p.alpha;
                    const long long off = (long long)row * p.ldc + col;
                    if (split) {  // partial sum of a K range; bias from split 0
                        if (p.bias && blockIdx.z == 0) x += p.bias[col];
                        atomicAdd(static_cast<float*>(p.C) + off, x);
                        continue;
                    }
                    if (p.bias) x += p.bias[col];
                    if (p.relu) x = fmaxf(x, 0.0f);
                    if (p.c_bf16) {
                        __nv_bfloat16* C = static_cast<__nv_bfloat16*>(p.C);
                        C[off] = __float2bfloat16(x);
                    } else {
                        float* C = static_cast<float*>(p.C);
                        C[off] = p.accumulate ? C[off] + x : x;
                    }
                }
            }
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(128) tc_gemm_kernel(GemmArgs p) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[kStages + 1];
    __shared__ uint32_t tmem_slot;
    constexpr int kABytes = kBM * kBK * 2;
    constexpr int kBBytes = BN * kBK * 2;
    constexpr int kStageBytes = kABytes + kBBytes;
    constexpr uint32_t kIdesc = idesc_bf16(kBM, BN);

    const int warp = threadIdx.x >> 5;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
    // 1024-byte aligned base (the swizzle atoms); the launch adds 1 KiB slack
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    // split-K: this CTA reduces K tiles [kt0, kt0 + nk)
    const int nk_total = (p.K + kBK - 1) / kBK;
    const bool split = p.k_tiles_per_split > 0;
    const int kt0 = split ? blockIdx.z * p.k_tiles_per_split : 0;
    const int nk = split ? max(0, min(p.k_tiles_per_split, nk_total - kt0)) : nk_total;
    const int k_base = kt0 * kBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s <= kStages; ++s) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    // prologue: stages 0 .. kStages-2
#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) {
            const uint32_t sa = sbase + s * kStageBytes;
            stage_tile<kBM>(sa, p.A, p.lda, m0, p.M, k_base + s * kBK, p.K);
            stage_tile<BN>(sa + kABytes, p.B, p.ldb, n0, p.N, k_base + s * kBK, p.K);
        }
        cp_async_commit();
    }

    bool ok = true;
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % kStages;
        cp_async_wait<kStages - 2>();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        // block-uniform: a timed-out wait anywhere ends the loop for all threads
        ok = __syncthreads_and(ok);
        if (!ok) break;
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t sa = sbase + s * kStageBytes;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
                // K = 16 per instruction: 32 bytes further into every 128-byte row
                const uint64_t ad = kmajor_sw128_desc(sa + kk * 32);
                const uint64_t bd = kmajor_sw128_desc(sa + kABytes + kk * 32);
                umma_bf16(tmem, ad, bd, kIdesc, (kt > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(smem_u32(&bars[s]));
        }
        // prefetch tile kt + kStages - 1 into the stage the previous MMAs used
        const int kn = kt + kStages - 1;
        if (kn < nk) {
            const int sn = kn % kStages;
            if (kt >= 1) ok = mbar_wait(smem_u32(&bars[sn]), ((kt - 1) / kStages) & 1);
            if (ok) {
                const uint32_t sa = sbase + sn * kStageBytes;
                stage_tile<kBM>(sa, p.A, p.lda, m0, p.M, k_base + kn * kBK, p.K);
                stage_tile<BN>(sa + kABytes, p.B, p.ldb, n0, p.N, k_base + kn * kBK, p.K);
            }
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
    ok = __syncthreads_and(ok);
    // the last commit completes after every MMA of the tile
    if (ok && nk > 0) ok = mbar_wait(smem_u32(&bars[(nk - 1) % kStages]), ((nk - 1) / kStages) & 1);
    ok = __syncthreads_and(ok);
    if (!ok && threadIdx.x == 0) atomicExch(p.error, 1);
    tc_fence_after();

    if (ok) gemm_epilogue<BN>(p, tmem, m0, n0, nk > 0, split);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// TMA + warp-specialised variant (the default).  Warp 0's lane 0 is the
// producer: per K tile it waits for the stage to be free (the MMAs that read
// it committed to empty[s]), posts the stage's byte count on full[s] and
// issues two cp.async.bulk.tensor loads (A 128 x 64, B BN x 64) that the
// tensor-map hardware writes in the 128-byte-swizzled layout, zero-filling
// rows and K beyond the matrix.  Warp 1's lane 0 issues the MMAs when full[s]
// completes and commits them to empty[s].  The last commit goes to `done`;
// then all four warps run the epilogue.  Every wait is bounded: on a timeout
// the error word is set, loads already issued are waited for (bounded) and
// the tensor memory is freed.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// MSUB 128-row sub-tiles of A per CTA (1 or 2): with 2, a CTA computes a
// 256 x BN tile as two M = 128 accumulators that share every staged B tile,
// which cuts the operand bytes moved per FLOP by a third at BN = 256.
template <int BN, int MSUB = 1>
struct TmaStages {
    static constexpr int kStageBytes = MSUB * kBM * kBK * 2 + BN * kBK * 2;
    static constexpr int value = (196608 / kStageBytes) < 8 ? (196608 / kStageBytes) : 8;
};

template <int BN, int MSUB>
__global__ void __launch_bounds__(128) tc_gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                          const __grid_constant__ CUtensorMap tmB,
                                                          GemmArgs p) {
    constexpr int S = TmaStages<BN, MSUB>::value;
    constexpr int kABytes = MSUB * kBM * kBK * 2;
    constexpr int kStageBytes = TmaStages<BN, MSUB>::kStageBytes;
    constexpr int kCols = MSUB * BN;  // tensor-memory columns of the accumulators
    constexpr uint32_t kIdesc = idesc_bf16(kBM, BN);
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t empty[S];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_err, s_consumed;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kBM * MSUB, n0 = blockIdx.x * BN;
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    const int nk_total = (p.K + kBK - 1) / kBK;
    const bool split = p.k_tiles_per_split > 0;
    const int kt0 = split ? blockIdx.z * p.k_tiles_per_split : 0;
    const int nk = split ? max(0, min(p.k_tiles_per_split, nk_total - kt0)) : nk_total;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(smem_u32(&full[i]), 1);
            mbar_init(smem_u32(&empty[i]), 1);
        }
        mbar_init(smem_u32(&done), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s_err = 0;
        s_consumed = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    volatile int* err = &s_err;

    int issued = 0;
    if (warp == 0 && lane == 0) {
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % S;
            if (kt >= S && !mbar_wait(smem_u32(&empty[s]), ((kt / S) - 1) & 1)) {
                *err = 1;
                break;
            }
            if (*err) break;
            const uint32_t sa = sbase + s * kStageBytes;
            const int kx = (kt0 + kt) * kBK;
            mbar_expect_tx(smem_u32(&full[s]), kStageBytes);
            tma_load_2d(sa, &tmA, kx, m0, smem_u32(&full[s]));
            tma_load_2d(sa + kABytes, &tmB, kx, n0, smem_u32(&full[s]));
            ++issued;
        }
    } else if (warp == 1 && lane == 0) {
        int kt = 0;
        for (; kt < nk; ++kt) {
            const int s = kt % S;
            if (!mbar_wait(smem_u32(&full[s]), (kt / S) & 1)) {
                *err = 1;
                break;
            }
            tc_fence_after();
            const uint32_t sa = sbase + s * kStageBytes;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
                const uint64_t bd = kmajor_sw128_desc(sa + kABytes + kk * 32);
#pragma unroll
                for (int m = 0; m < MSUB; ++m) {
                    // sub-tile m: rows 128m.. of the staged A (128 B per row)
                    const uint64_t ad = kmajor_sw128_desc(sa + m * kBM * 128 + kk * 32);
                    umma_bf16(tmem + m * BN, ad, bd, kIdesc, (kt > 0 || kk > 0) ? 1u : 0u);
                }
            }
            umma_commit(smem_u32(&empty[s]));
        }
        s_consumed = kt;
        umma_commit(smem_u32(&done));  // arrives once every MMA issued above has completed
    }
    __syncthreads();
    bool ok = (*err == 0);
    // all MMAs (and with them every read of the staged tiles) are complete
    if (nk > 0 && !mbar_wait(smem_u32(&done), 0)) ok = false;
    ok = __syncthreads_and(ok);
    if (warp == 0 && lane == 0) {
        // loads issued but never consumed (only after a timeout) must land
        // before the CTA's shared memory is released
        for (int kt = s_consumed; kt < issued; ++kt) mbar_wait(smem_u32(&full[kt % S]), (kt / S) & 1);
    }
    __syncwarp();
    if (!ok && threadIdx.x == 0) atomicExch(p.error, 1);
    tc_fence_after();
    if (ok) {
#pragma unroll
        for (int m = 0; m < MSUB; ++m)
            gemm_epilogue<BN>(p, tmem + m * BN, m0 + m * kBM, n0, nk > 0, split);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols)
                     : "memory");
    }
}

// 2-D bf16 map of a row-major [rows][ld] matrix with K = cols valid columns:
// boxes of 64 K elements (128 bytes) x box_rows rows, 128-byte swizzle,
// zero fill outside.
bool make_kmajor_map(CUtensorMap* map, const void* base, int rows, int cols, int ld, int box_rows) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int MSUB>
int launch_gemm_tma(const GemmArgs& p, cudaStream_t s, bool* used) {
    *used = false;
    CUtensorMap ta, tb;
    if (!make_kmajor_map(&ta, p.A, p.M, p.K, p.lda, kBM * MSUB) ||
        !make_kmajor_map(&tb, p.B, p.N, p.K, p.ldb, BN))
        return DGC_OK;
    const int smem = TmaStages<BN, MSUB>::value * TmaStages<BN, MSUB>::kStageBytes + 1024;
    static std::atomic<unsigned long long> configured{0};
    const int rc = once_per_device(configured, [smem]() -> int {
        DGC_CUDA(cudaFuncSetAttribute(tc_gemm_tma_kernel<BN, MSUB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return DGC_OK;
    });
    if (rc != DGC_OK) return rc;
    const int splits = p.k_tiles_per_split > 0
                           ? ceil_div(ceil_div(p.K, kBK), p.k_tiles_per_split) : 1;
    const dim3 grid(ceil_div(p.N, BN), ceil_div(p.M, kBM * MSUB), splits);
    DGC_TRACE("tc_gemm_tma_kernel", s);
    tc_gemm_tma_kernel<BN, MSUB><<<grid, 128, smem, s>>>(ta, tb, p);
    DGC_LAUNCH_CHECK("tc_gemm_tma_kernel");
    *used = true;
    return DGC_OK;
}

template <int BN>
int launch_gemm(const GemmArgs& p, cudaStream_t s) {
    const int smem = kStages * (kBM * kBK * 2 + BN * kBK * 2) + 1024;
    static std::atomic<unsigned long long> configured{0};
    const int rc = once_per_device(configured, [smem]() -> int {
        DGC_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
        return DGC_OK;
    });
    if (rc != DGC_OK) return rc;
    const int splits = p.k_tiles_per_split > 0
                           ? ceil_div(ceil_div(p.K, kBK), p.k_tiles_per_split) : 1;
    const dim3 grid(ceil_div(p.N, BN), ceil_div(p.M, kBM), splits);
    DGC_TRACE("tc_gemm_kernel", s);
    tc_gemm_kernel<BN><<<grid, 128, smem, s>>>(p);
    DGC_LAUNCH_CHECK("tc_gemm_kernel");
    return DGC_OK;
}

}  // namespace

int tc_gemm(const GemmArgs& p, cudaStream_t s) {
    const int splits = p.k_tiles_per_split > 0 ? ceil_div(ceil_div(p.K, kBK), p.k_tiles_per_split) : 1;
    // 256-column tiles halve the B traffic per FLOP; used when they still
    // give every SM a tile
    const int bn = p.N <= 64 ? 64
                   : (p.N > 128 && (long long)ceil_div(p.M, kBM) * ceil_div(p.N, 256) * splits >= 148)
                       ? 256
                       : 128;
    // DGC_GEMM=cpasync selects the cp.async pipeline (also the fallback when
    // the driver cannot encode tensor maps)
    const char* e = std::getenv("DGC_GEMM");
    if (!(e && std::strcmp(e, "cpasync") == 0)) {
        // 256 x 256 tiles (two accumulators) where they still give every SM a tile
        const bool two = bn == 256 &&
                         (long long)ceil_div(p.M, 2 * kBM) * ceil_div(p.N, 256) * splits >= 148;
        bool used = false;
        int rc = bn == 64    ? launch_gemm_tma<64, 1>(p, s, &used)
                 : two       ? launch_gemm_tma<256, 2>(p, s, &used)
                 : bn == 256 ? launch_gemm_tma<256, 1>(p, s, &used)
                             : launch_gemm_tma<128, 1>(p, s, &used);
        if (rc != DGC_OK || used) return rc;
    }
    if (bn == 64) return launch_gemm<64>(p, s);
    if (bn == 256) return launch_gemm<256>(p, s);
    return launch_gemm<128>(p, s);
}

}  // namespace dgc
