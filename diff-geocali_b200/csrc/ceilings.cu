// ceilings.cu -- measurement kernels: the ceilings the gather-bound kernels
// of this library are measured against (no counterpart in the reference).
//
// The ray-marching projector and the voxel-driven backprojector spend their
// time in 16-byte loads whose lines are mostly served by the SM's L1 (the
// forward's 32 lanes are 32 detector rows of one column and sample nearly
// contiguous z-fastest quads) or by L2, not by HBM.  Their algorithmic bytes
// per second are therefore compared with what the SMs can pull through L1 and
// L2 with 16-byte loads at all, measured here on the same GPU:
//
//   * gather_ceiling_kernel: every warp issues independent 16-byte loads, one
//     float4 per lane, a warp covering 512 contiguous bytes (four 128-byte
//     lines) per load -- the best case for 16 bytes per lane -- or, with a
//     lane stride above one element, the wider spread of the backprojector's
//     loads (lanes ~1.7 quads apart: seven lines per load).  With a small
//     window shared by all CTAs the lines stay in each SM's L1 (the L1
//     ceiling); with every CTA ranging over one buffer far larger
//     than an SM's L1 but smaller than L2, in a random line order, nearly
//     every load misses L1 and hits L2 (the L2-to-SM ceiling).
//   * issue_ceiling_kernel: eight independent FFMA chains per thread, the
//     rate at which the SMs retire warp instructions.
//
// Bytes are counted as the kernels count theirs: 16 per lane and load.
#include "common.cuh"

namespace dgc {
namespace {

constexpr int kGatherThreads = 256;
constexpr int kGatherUnroll = 8;

// window_mask + 1 = elements (float4) the loads range over, a power of two
// >= 64, one window shared by all CTAs.  Each load of warp w reads, lane l,
// element g*64 + floor(l * stride16 / 16) of the window -- stride16 = 16: 32
// contiguous elements (512 bytes); 27: lanes 1.6875 elements apart, the
// backprojector's pattern at magnification 1.67 -- the 1 KiB group g drawn
// by a linear congruential sequence per warp, so consecutive loads of a warp
// touch unrelated lines.
__global__ void __launch_bounds__(kGatherThreads)
gather_ceiling_kernel(const float4* __restrict__ base, unsigned window_mask, int iterations,
                      unsigned stride16, float* sink) {
    const unsigned lane = ((threadIdx.x & 31) * stride16) >> 4;
    const unsigned warp = (blockIdx.x * (kGatherThreads / 32)) + (threadIdx.x >> 5);
    unsigned h = warp * 2654435761u + 12345u;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = 0; i < iterations; i += kGatherUnroll) {
        float4 q[kGatherUnroll];
#pragma unroll
        for (int u = 0; u < kGatherUnroll; ++u) {
            h = h * 1664525u + 1013904223u;
            q[u] = __ldg(base + ((((h >> 8) << 6) + lane) & window_mask));
        }
#pragma unroll
        for (int u = 0; u < kGatherUnroll; ++u) {
            acc.x += q[u].x;
            acc.y += q[u].y;
            acc.z += q[u].z;
            acc.w += q[u].w;
        }
    }
    const float s = acc.x + acc.y + acc.z + acc.w;
    if (s == 1234.5f) sink[0] = s;  // keeps the loads live; never true for the zeroed input
}

constexpr int kIssueThreads = 256;

__global__ void __launch_bounds__(kIssueThreads)
issue_ceiling_kernel(int iterations, float seed, float* sink) {
    float a0 = seed, a1 = seed + 1.f, a2 = seed + 2.f, a3 = seed + 3.f;
    float a4 = seed + 4.f, a5 = seed + 5.f, a6 = seed + 6.f, a7 = seed + 7.f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, m, c);
            a1 = fmaf(a1, m, c);
            a2 = fmaf(a2, m, c);
            a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c);
            a5 = fmaf(a5, m, c);
            a6 = fmaf(a6, m, c);
            a7 = fmaf(a7, m, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 1234.5f) sink[0] = s;
}

int sm_count(int* out) {
    int dev = 0;
    DGC_CUDA(cudaGetDevice(&dev));
    DGC_CUDA(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
    return DGC_OK;
}

}  // namespace
}  // namespace dgc

extern "C" int dgc_ceiling_gather(const void* buffer, size_t buffer_bytes, int level, int iterations,
                                  int ctas_per_sm, int lane_stride16, float* sink, double* bytes,
                                  void* stream) {
    using namespace dgc;
    clear_error();
    DGC_REQUIRE(buffer && sink && bytes, "pointers must be non-null");
    DGC_REQUIRE(level == 1 || level == 2, "level must be 1 (L1-resident) or 2 (L2-resident)");
    DGC_REQUIRE(iterations > 0 && iterations % kGatherUnroll == 0,
                "iterations must be a positive multiple of 8");
    DGC_REQUIRE(ctas_per_sm > 0 && ctas_per_sm <= 8, "ctas_per_sm must be in [1, 8]");
    DGC_REQUIRE(((uintptr_t)buffer & 15u) == 0, "buffer must be 16-byte aligned");
    DGC_REQUIRE(lane_stride16 >= 16 && lane_stride16 <= 32,
                "lane_stride16 must be in [16, 32] (lanes 1 to 2 elements apart)");
    int sms = 0;
    int rc = sm_count(&sms);
    if (rc != DGC_OK) return rc;
    const long long grid = (long long)sms * ctas_per_sm;
    const long long elems = (long long)(buffer_bytes / 16);
    unsigned window = 0;
    if (level == 1) {
        window = 2048;  // 32 KiB: resident in each SM's L1
        DGC_REQUIRE(elems >= window, "buffer must hold at least 32 KiB");
    } else {
        // the largest power of two of 16-byte elements in the buffer; it
        // should be far larger than an SM's L1 and fit in L2 (16-96 MiB)
        window = 1u;
        while ((long long)window * 2 <= elems && window < (1u << 30)) window *= 2;
        DGC_REQUIRE(window >= (1u << 20), "the L2 case needs a buffer of at least 16 MiB");
    }
    {
        DGC_TRACE("gather_ceiling_kernel", (cudaStream_t)stream);
        gather_ceiling_kernel<<<(unsigned)grid, kGatherThreads, 0, (cudaStream_t)stream>>>(
            static_cast<const float4*>(buffer), window - 1u, iterations, (unsigned)lane_stride16,
            sink);
        DGC_LAUNCH_CHECK("gather_ceiling_kernel");
    }
    *bytes = (double)grid * kGatherThreads * (double)iterations * 16.0;
    return DGC_OK;
}

extern "C" int dgc_ceiling_issue(int iterations, int ctas_per_sm, float* sink,
                                 double* warp_instructions, void* stream) {
    using namespace dgc;
    clear_error();
    DGC_REQUIRE(sink && warp_instructions, "pointers must be non-null");
    DGC_REQUIRE(iterations > 0, "iterations must be positive");
    DGC_REQUIRE(ctas_per_sm > 0 && ctas_per_sm <= 8, "ctas_per_sm must be in [1, 8]");
    int sms = 0;
    int rc = sm_count(&sms);
    if (rc != DGC_OK) return rc;
    const long long grid = (long long)sms * ctas_per_sm;
    {
        DGC_TRACE("issue_ceiling_kernel", (cudaStream_t)stream);
        issue_ceiling_kernel<<<(unsigned)grid, kIssueThreads, 0, (cudaStream_t)stream>>>(
            iterations, 1.0f, sink);
        DGC_LAUNCH_CHECK("issue_ceiling_kernel");
    }
    // 128 FFMA per iteration and thread; the loop's own instructions are
    // left out, so the figure is a slight underestimate of the issue rate
    *warp_instructions = (double)grid * (kIssueThreads / 32) * (double)iterations * 128.0;
    return DGC_OK;
}
