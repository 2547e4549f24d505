// nn_kernels.cu -- data movement around the tensor-core GEMM for the
// convolution layers of the warm-start network (NHWC activations).
// No counterpart in the reference.
//
//   im2col:  col[(b*Ho + oy)*Wo + ox][(ky*kw + kx)*C + c] = x[b][oy*s - p + ky][ox*s - p + kx][c]
//            (zero outside the image and for k >= kh*kw*C up to the padded width Kp)
//   col2im:  the adjoint, as a gather per input element (no atomics).
#include <cuda_bf16.h>

#include "common.cuh"

namespace dgc {
namespace {

__global__ void im2col_nhwc_kernel(const __nv_bfloat16* __restrict__ x, int B, int H, int W, int C,
                                   int kh, int kw, int stride, int pad, int Ho, int Wo,
                                   __nv_bfloat16* __restrict__ col, int Kp, bool vec8) {
    const long long rows = (long long)B * Ho * Wo;
    const int kchunks = vec8 ? Kp / 8 : Kp;
    const long long total = rows * kchunks;
    const int Kreal = kh * kw * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = i / kchunks;
        const int kc = (int)(i - m * kchunks);
        const int k = vec8 ? kc * 8 : kc;
        const int ox = (int)(m % Wo);
        const long long t = m / Wo;
        const int oy = (int)(t % Ho);
        const int b = (int)(t / Ho);
        const int tap = k / C, c = k - tap * C;
        const int ky = tap / kw, kx = tap - ky * kw;
        const int iy = oy * stride - pad + ky, ix = ox * stride - pad + kx;
        const bool inside = k < Kreal && iy >= 0 && iy < H && ix >= 0 && ix < W;
        const long long src = (((long long)b * H + iy) * W + ix) * C + c;
        if (vec8) {
            uint4 v = make_uint4(0, 0, 0, 0);
            if (inside) v = *reinterpret_cast<const uint4*>(x + src);
            *reinterpret_cast<uint4*>(col + m * Kp + k) = v;
        } else {
            col[m * Kp + k] = inside ? x[src] : __float2bfloat16(0.0f);
        }
    }
}

__global__ void col2im_nhwc_kernel(const float* __restrict__ col, int B, int H, int W, int C,
                                   int kh, int kw, int stride, int pad, int Ho, int Wo, int Kp,
                                   float* __restrict__ dx) {
    const long long total = (long long)B * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int ix = (int)(t % W);
        t /= W;
        const int iy = (int)(t % H);
        const int b = (int)(t / H);
        float acc = 0.0f;
        for (int ky = 0; ky < kh; ++ky) {
            const int ny = iy + pad - ky;
            if (ny < 0 || ny % stride) continue;
            const int oy = ny / stride;
            if (oy >= Ho) continue;
            for (int kx = 0; kx < kw; ++kx) {
                const int nx = ix + pad - kx;
                if (nx < 0 || nx % stride) continue;
                const int ox = nx / stride;
                if (ox >= Wo) continue;
                const long long m = ((long long)b * Ho + oy) * Wo + ox;
                acc += col[m * Kp + (ky * kw + kx) * C + c];
            }
        }
        dx[i] = acc;
    }
}

int conv_out(int n, int k, int stride, int pad) { return (n + 2 * pad - k) / stride + 1; }

}  // namespace
}  // namespace dgc

using namespace dgc;

extern "C" int dgc_im2col_nhwc_bf16(const void* x, int B, int H, int W, int C, int kh, int kw,
                                    int stride, int pad, void* col, int Kp, void* stream) {
    clear_error();
    DGC_REQUIRE(x && col, "x and col must be non-null");
    DGC_REQUIRE(B > 0 && H > 0 && W > 0 && C > 0 && kh > 0 && kw > 0 && stride > 0 && pad >= 0,
                "invalid convolution shape");
    DGC_REQUIRE(Kp >= kh * kw * C, "Kp must be >= kh*kw*C");
    const int Ho = conv_out(H, kh, stride, pad), Wo = conv_out(W, kw, stride, pad);
    DGC_REQUIRE(Ho > 0 && Wo > 0, "empty convolution output");
    cudaStream_t s = (cudaStream_t)stream;
    DGC_TRACE("im2col_nhwc", s);
    const bool vec8 = (C % 8 == 0) && (Kp % 8 == 0) && ((uintptr_t)x % 16 == 0) &&
                      ((uintptr_t)col % 16 == 0);
    const long long total = (long long)B * Ho * Wo * (vec8 ? Kp / 8 : Kp);
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    im2col_nhwc_kernel<<<blocks, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(x), B, H, W, C, kh,
                                              kw, stride, pad, Ho, Wo,
                                              static_cast<__nv_bfloat16*>(col), Kp, vec8);
    DGC_LAUNCH_CHECK("im2col_nhwc");
    return DGC_OK;
}

extern "C" int dgc_col2im_nhwc_f32(const float* col, int B, int H, int W, int C, int kh, int kw,
                                   int stride, int pad, int Kp, float* dx, void* stream) {
    clear_error();
    DGC_REQUIRE(col && dx, "col and dx must be non-null");
    DGC_REQUIRE(B > 0 && H > 0 && W > 0 && C > 0 && kh > 0 && kw > 0 && stride > 0 && pad >= 0,
                "invalid convolution shape");
    DGC_REQUIRE(Kp >= kh * kw * C, "Kp must be >= kh*kw*C");
    const int Ho = conv_out(H, kh, stride, pad), Wo = conv_out(W, kw, stride, pad);
    DGC_REQUIRE(Ho > 0 && Wo > 0, "empty convolution output");
    cudaStream_t s = (cudaStream_t)stream;
    DGC_TRACE("col2im_nhwc", s);
    const long long total = (long long)B * H * W * C;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    col2im_nhwc_kernel<<<blocks, 256, 0, s>>>(col, B, H, W, C, kh, kw, stride, pad, Ho, Wo, Kp, dx);
    DGC_LAUNCH_CHECK("col2im_nhwc");
    return DGC_OK;
}
