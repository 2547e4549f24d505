// preprocess.cu -- raw detector frames to line integrals in the operators'
// [A,U,V] layout: dark/flat-field correction, -log, and the [A,V,U] -> [A,U,V]
// transpose in one pass.  The reference requires this upstream of its
// operators (README.md:97, README.md:108; docs/USAGE.md:247-251 transposes
// [A,V,U] data with permute(0,2,1)); it ships no code for it.
//
//   p[a,u,v] = -log(max((raw - dark) / (flat - dark), min_ratio))
//
// with dark = 0 and flat = 1 where not given.  Frames stored [A,V,U] (U
// fastest, the usual detector readout) are transposed through 32 x 33
// shared-memory tiles so that both the reads (along U) and the writes (along
// V) are coalesced; [A,U,V] input is processed in place of layout.
#include <cmath>

#include "common.cuh"

namespace dgc {
namespace {

__device__ __forceinline__ float line_integral(float raw, float dark, float flat, float min_ratio) {
    const float ratio = __fdiv_rn(raw - dark, flat - dark);
    // NaN (0/0) and anything below min_ratio take min_ratio
    return -logf(ratio >= min_ratio ? ratio : min_ratio);
}

// grid: (ceil(U/32), ceil(V/32), A); block (32, 8)
__global__ void preprocess_avu_kernel(const float* __restrict__ raw, const float* __restrict__ dark,
                                      const float* __restrict__ flat, int A, int U, int V,
                                      float min_ratio, float* __restrict__ out) {
    __shared__ float tile[32][33];
    const int a = blockIdx.z;
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const float* frame = raw + (long long)a * V * U;
    for (int j = ty; j < 32; j += 8) {
        const int v = v0 + j, u = u0 + tx;
        if (v < V && u < U) {
            const long long i = (long long)v * U + u;
            tile[j][tx] = line_integral(frame[i], dark ? dark[i] : 0.0f, flat ? flat[i] : 1.0f,
                                        min_ratio);
        }
    }
    __syncthreads();
    float* dst = out + (long long)a * U * V;
    for (int j = ty; j < 32; j += 8) {
        const int u = u0 + j, v = v0 + tx;
        if (u < U && v < V) dst[(long long)u * V + v] = tile[tx][j];
    }
}

__global__ void preprocess_auv_kernel(const float* __restrict__ raw, const float* __restrict__ dark,
                                      const float* __restrict__ flat, int A, int U, int V,
                                      float min_ratio, float* __restrict__ out) {
    const long long frame = (long long)U * V;
    const long long total = frame * A;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long f = i % frame;
        out[i] = line_integral(raw[i], dark ? dark[f] : 0.0f, flat ? flat[f] : 1.0f, min_ratio);
    }
}

}  // namespace
}  // namespace dgc

using namespace dgc;

extern "C" int dgc_preprocess(const float* raw, const float* dark, const float* flat, int A, int U,
                              int V, int layout_avu, float min_ratio, float* out, void* stream) {
    clear_error();
    DGC_REQUIRE(raw && out, "raw and out must be non-null");
    DGC_REQUIRE(A > 0 && U > 0 && V > 0, "A, U and V must be positive");
    DGC_REQUIRE(A <= 65535, "A exceeds the 65535 frames of one launch");
    DGC_REQUIRE(std::isfinite(min_ratio) && min_ratio > 0.0f, "min_ratio must be positive and finite");
    DGC_REQUIRE(raw != out, "out must not alias raw");
    cudaStream_t s = (cudaStream_t)stream;
    DGC_TRACE("preprocess", s);
    if (layout_avu) {
        const dim3 grid((unsigned)ceil_div(U, 32), (unsigned)ceil_div(V, 32), (unsigned)A);
        preprocess_avu_kernel<<<grid, dim3(32, 8), 0, s>>>(raw, dark, flat, A, U, V, min_ratio, out);
    } else {
        const long long total = (long long)A * U * V;
        const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
        preprocess_auv_kernel<<<blocks, 256, 0, s>>>(raw, dark, flat, A, U, V, min_ratio, out);
    }
    DGC_LAUNCH_CHECK("preprocess");
    return DGC_OK;
}
