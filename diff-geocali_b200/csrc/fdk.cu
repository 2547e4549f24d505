// fdk.cu -- FDK ramp filtering for sm_100a.
//
// The reference (TomSHINING/diff-geoCali, cbct_backprojector/filtering.py:54-104)
// cosine-weights the projections, zero-pads U to P = 2^bitlen(2U-1), multiplies
// the FFT along U by Re(FFT(discrete Ram-Lak)) x Hann, inverse-transforms,
// crops and scales by pixel*sid/sod.  With that padding the circular
// convolution never wraps onto the data, and the filter response is real and
// even, so the whole filter is the symmetric Toeplitz product
//
//     y[a,u,v] = sum_k h[|u-k|] * w[a,k,v],   u,k in [0,U)
//
// i.e. per view a (U x U) * (U x V) matrix product with a Toeplitz left
// factor.  This file evaluates it as one register-blocked FP32 product per
// (view, 128x128 output tile): the cosine weight is applied while the input
// tile is staged into shared memory, the Toeplitz factor is generated from a
// sliding window of taps, and the pixel*sid/sod scale is applied in the
// epilogue.  No FFT, no complex temporaries, no padding buffer.
#include "common.cuh"
#include "fdk.cuh"

#include <cmath>
#include <cstddef>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace dgc {

// ---------------------------------------------------------------------------
// Filter taps (host, FP64)
// ---------------------------------------------------------------------------

// h[m], m in [0, U): inverse DFT of H[k] = R[k] * hann[k], with R the DFT of
// the discrete Ram-Lak kernel r[0] = 1/(4 px^2), r[n odd] = -1/(pi n px)^2
// (n taken in (-P/2, P/2]), and hann[k] = 0.5 + 0.5 cos(2 pi f_k / alpha) for
// |f_k| <= alpha/2 (f_k the DFT bin frequency in cycles/sample), else 0.
// Direct sums over the even symmetry; cached per (U, px, alpha).
int fdk_taps_host(int U, double px, double alpha, std::vector<double>& out) {
    static std::mutex mu;
    static std::map<std::tuple<int, double, double>, std::vector<double>> cache;
    const auto key = std::make_tuple(U, px, alpha);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            out = it->second;
            return DGC_OK;
        }
    }
    int bl = 0;
    for (int n = 2 * U - 1; n; n >>= 1) ++bl;
    const int P = 1 << bl;
    std::vector<double> cs(P);
    for (int j = 0; j < P; ++j) cs[j] = std::cos(2.0 * M_PI * (double)j / (double)P);
    // R[k] for k in [0, P/2] (R is even in k).
    const int half = P / 2;
    std::vector<double> Hk(half + 1);
    for (int k = 0; k <= half; ++k) {
        double R = 1.0 / (4.0 * px * px);
        // odd n in (0, P/2) appear twice (n and -n); n = P/2 once when odd.
        for (int n = 1; n <= half; n += 2) {
            const double rn = -1.0 / ((M_PI * n * px) * (M_PI * n * px));
            const double weight = (n == half) ? 1.0 : 2.0;
            R += weight * rn * cs[((long long)k * n) % P];
        }
        const double f = (k == half) ? -0.5 : (double)k / (double)P;
        const double hann =
            std::fabs(f) <= alpha * 0.5 ? 0.5 + 0.5 * std::cos(2.0 * M_PI * f / alpha) : 0.0;
        Hk[k] = R * hann;
    }
    out.assign(U, 0.0);
    for (int m = 0; m < U; ++m) {
        double acc = Hk[0];
        for (int k = 1; k < half; ++k) acc += 2.0 * Hk[k] * cs[((long long)k * m) % P];
        acc += Hk[half] * cs[((long long)half * m) % P];
        out[m] = acc / P;
    }
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = out;
    return DGC_OK;
}

// ---------------------------------------------------------------------------
// Filter kernel
// ---------------------------------------------------------------------------

constexpr int FBM = 128;  // output rows (U) per CTA
constexpr int FBN = 128;  // output columns (V) per CTA
constexpr int FBK = 16;   // reduction slice

// ADJ = false: y = c H(w P) (the filter).  ADJ = true: its adjoint, z = H(g)
// for the upstream gradient g (H is symmetric), grad P = c w z, and per CTA
// the FP64 sums of g*y, z*P*dw/dD and (CG, the frame centre's gradients
// asked for) z*P*u_c/dist^3, z*P*v_c/dist^3 -- zeros without CG -- for the
// distance and centre gradients; c = pixel*sid/sod,
// w = D/dist the cosine weight with D the source's distance to the detector
// plane (sid unless a frame is given), u_c, v_c the pixel's offsets from the
// frame centre in length units, dist^2 = D^2 + u_c^2 + v_c^2, and
// dw/dD = (u_c^2 + v_c^2)/dist^3.
template <bool ADJ, bool CG = false>
__global__ void __launch_bounds__(256, 2) fdk_filter_kernel(FdkArgs p) {
    __shared__ __align__(16) float ws[FBK][FBN];
    __shared__ f32x2 gw2[FBM + FBK];  // taps, each duplicated into a packed pair
    __shared__ double s_part[8][kFdkPartials];
    const int a = blockIdx.z;
    const int m0 = blockIdx.y * FBM;
    const int n0 = blockIdx.x * FBN;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const float sid = p.sid[a], sod = p.sod[a];
    const float dn = p.frame_dist ? p.frame_dist[a] : sid;  // preweight distance D
    const float dn2 = dn * dn;
    const float* __restrict__ Pa = p.projections + (long long)a * p.U * p.V;
    const float* __restrict__ Ga = ADJ ? p.grad_filtered + (long long)a * p.U * p.V : nullptr;
    const float cu = p.frame_u ? p.frame_u[a] : 0.5f * (p.U - 1);
    const float cv = p.frame_v ? p.frame_v[a] : 0.5f * (p.V - 1);

    // 8 x 8 outputs per thread as packed pairs along v: one fma.rn.f32x2 per
    // two outputs (lane by lane the scalar FMA, in the same order)
    f32x2 acc2[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc2[i][j] = pack2(0.0f, 0.0f);

    for (int k0 = 0; k0 < p.U; k0 += FBK) {
        {   // stage the cosine-weighted input slice w[k0..k0+FBK) x [n0..n0+FBN)
            const int r = tid >> 4;
            const int k = k0 + r;
            const int c0 = (tid & 15) * 8;
            const float uu = ((float)k - cu) * p.pixel_size;
            const float wk = (p.uweight && k < p.U) ? p.uweight[(long long)a * p.U + k] : 1.0f;
            float vals[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int v = n0 + c0 + j;
                float val = 0.0f;
                if (k < p.U && v < p.V) {
                    if (ADJ) {
                        val = Ga[(long long)k * p.V + v];
                    } else {
                        const float vv = ((float)v - cv) * p.pixel_size;
                        const float dist = sqrtf(dn2 + uu * uu + vv * vv);
                        val = Pa[(long long)k * p.V + v] * (dn / dist) * wk;
                    }
                }
                vals[j] = val;
            }
            *reinterpret_cast<float4*>(&ws[r][c0]) = make_float4(vals[0], vals[1], vals[2], vals[3]);
            *reinterpret_cast<float4*>(&ws[r][c0 + 4]) = make_float4(vals[4], vals[5], vals[6], vals[7]);
        }
        // Toeplitz window: gw[i] = h[|m0 - k0 - (FBK-1) + i|]
        for (int i = tid; i < FBM + FBK - 1; i += 256) {
            int d = m0 - k0 - (FBK - 1) + i;
            d = d < 0 ? -d : d;
            const float h = p.taps[min(d, p.U - 1)];
            gw2[i] = pack2(h, h);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < FBK; ++kk) {
            // a thread's columns: tx*4..+3 and FBN/2 + tx*4..+3, so the 16 lanes of
            // a load read contiguous 16-byte chunks (no bank conflicts)
            const ulonglong2 b0 = *reinterpret_cast<const ulonglong2*>(&ws[kk][tx * 4]);
            const ulonglong2 b1 = *reinterpret_cast<const ulonglong2*>(&ws[kk][FBN / 2 + tx * 4]);
            const f32x2 b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const f32x2 av = gw2[ty * 8 + i - kk + FBK - 1];
#pragma unroll
                for (int j = 0; j < 4; ++j) acc2[i][j] = fma2(av, b[j], acc2[i][j]);
            }
        }
        __syncthreads();
    }
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 e = unpack2(acc2[i][j]);
            acc[i][2 * j] = e.x;
            acc[i][2 * j + 1] = e.y;
        }
    // filtering.py:104: filtered * pixel_size * (sid / sod)
    const float ratio = sid / sod;
    if (!ADJ) {
        float* __restrict__ Oa = p.filtered + (long long)a * p.U * p.V;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int u = m0 + ty * 8 + i;
            if (u >= p.U) continue;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int v = n0 + (j < 4 ? tx * 4 + j : FBN / 2 + tx * 4 + j - 4);
                if (v < p.V) Oa[(long long)u * p.V + v] = (acc[i][j] * p.pixel_size) * ratio;
            }
        }
        return;
    }
    // adjoint epilogue: acc = z = H(g) at (u, v)
    const long long base = (long long)a * p.U * p.V;
    double s_gy = 0.0, s_zpw = 0.0, s_zpu = 0.0, s_zpv = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int u = m0 + ty * 8 + i;
        if (u >= p.U) continue;
        const float uu = ((float)u - cu) * p.pixel_size;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int v = n0 + (j < 4 ? tx * 4 + j : FBN / 2 + tx * 4 + j - 4);
            if (v >= p.V) continue;
            const long long idx = (long long)u * p.V + v;
            const float vv = ((float)v - cv) * p.pixel_size;
            const float r2 = uu * uu + vv * vv;
            const float dist = sqrtf(dn2 + r2);
            const float z = acc[i][j];
            if (p.grad_projections)
                p.grad_projections[base + idx] = (z * p.pixel_size) * ratio * (dn / dist);
            if (p.partials) {
                const double zp = (double)z * (double)Pa[idx];
                const double d3 = (double)dist * dist * dist;
                s_gy += (double)Ga[idx] * (double)p.forward_out[base + idx];
                s_zpw += zp * ((double)r2 / d3);
                if (CG) {
                    s_zpu += zp * ((double)uu / d3);
                    s_zpv += zp * ((double)vv / d3);
                }
            }
        }
    }
    if (!p.partials) return;
    // CTA sums in a fixed order: warp shuffles, then the eight warps in turn
    constexpr int kSums = CG ? 4 : 2;  // sums this variant accumulates
    s_gy = warp_sum(s_gy);
    s_zpw = warp_sum(s_zpw);
    if (CG) {
        s_zpu = warp_sum(s_zpu);
        s_zpv = warp_sum(s_zpv);
    }
    const int lane = tid & 31, warp = tid >> 5;
    if (lane == 0) {
        s_part[warp][0] = s_gy;
        s_part[warp][1] = s_zpw;
        if (CG) {
            s_part[warp][2] = s_zpu;
            s_part[warp][3] = s_zpv;
        }
    }
    __syncthreads();
    if (tid < kFdkPartials) {
        double t = 0.0;
        if (tid < kSums)
            for (int w8 = 0; w8 < 8; ++w8) t += s_part[w8][tid];
        const long long tiles = (long long)gridDim.x * gridDim.y;
        const long long tile = (long long)blockIdx.y * gridDim.x + blockIdx.x;
        p.partials[((long long)a * tiles + tile) * kFdkPartials + tid] = t;
    }
}

// Per view, from the CTA partials in a fixed order, with c = pixel*sid/sod:
//   dL/dsod = -sum(g y)/sod
//   dL/dsid = sum(g y)/sid + c sum(H(g) P dw/dD)   (D = sid: no frame distance)
//   dL/dD   = c sum(H(g) P dw/dD)                  (a frame distance D given)
//   dL/du   = c D pixel sum(H(g) P u_c/dist^3),  dL/dv likewise,
// u, v the frame centre (w = D/dist falls off away from it).
__global__ void fdk_distance_grads_kernel(const double* __restrict__ partials, long long tiles,
                                          FdkArgs p, FdkGrads g) {
    const int a = blockIdx.x;
    const int lane = threadIdx.x;  // one warp
    double s[kFdkPartials] = {0.0, 0.0, 0.0, 0.0};
    for (long long t = lane; t < tiles; t += 32) {
        const double* row = partials + ((long long)a * tiles + t) * kFdkPartials;
#pragma unroll
        for (int k = 0; k < kFdkPartials; ++k) s[k] += row[k];
    }
#pragma unroll
    for (int k = 0; k < kFdkPartials; ++k) s[k] = warp_sum(s[k]);
    if (lane == 0) {
        const double d_sid = p.sid[a], d_sod = p.sod[a];
        const double c = (double)p.pixel_size * (d_sid / d_sod);
        const double dn = p.frame_dist ? (double)p.frame_dist[a] : d_sid;
        const double gy = s[0], zpw = s[1];
        if (g.sid) g.sid[a] = (float)(p.frame_dist ? gy / d_sid : gy / d_sid + c * zpw);
        if (g.sod) g.sod[a] = (float)(-gy / d_sod);
        if (g.frame_dist) g.frame_dist[a] = (float)(c * zpw);
        if (g.frame_u) g.frame_u[a] = (float)(c * dn * (double)p.pixel_size * s[2]);
        if (g.frame_v) g.frame_v[a] = (float)(c * dn * (double)p.pixel_size * s[3]);
    }
}

// Parker's short-scan weights (D. L. Parker, Med. Phys. 9(2), 1982): for a
// scan over beta in [0, pi + 2*Gamma] and the fan angle gamma = atan(u_c/D)
// of detector column u (u_c = (u - (U-1)/2) * pixel and D = sid, or the
// preweight frame's centre and distance where one is given),
//   w = sin^2(pi/4 * beta / (Gamma - gamma))                 beta <  2(Gamma - gamma)
//   w = 1                                                   beta <= pi - 2 gamma
//   w = sin^2(pi/4 * (pi + 2 Gamma - beta) / (Gamma + gamma)) beta <= pi + 2 Gamma
// and 0 beyond, so that every ray and its conjugate (beta + pi + 2 gamma,
// -gamma) weigh 1 together.  Gamma is taken from the scan's own range,
// (range - pi) / 2, which must be at least the largest fan angle (Parker
// weights with a wider Gamma are the usual over-scan form).  beta runs from
// angles[0] in the direction of the scan; for a decreasing scan gamma flips
// sign with it.  FP64 (a table of A*U values).
__global__ void parker_weights_kernel(const float* __restrict__ angles,
                                      const float* __restrict__ sid,
                                      const float* __restrict__ frame_dist,
                                      const float* __restrict__ frame_u, int A, int U, float px,
                                      float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)A * U) return;
    const int a = (int)(i / U), u = (int)(i - (long long)a * U);
    const double b0 = angles[0], bl = angles[A - 1];
    const double dir = bl >= b0 ? 1.0 : -1.0;
    const double beta = dir * ((double)angles[a] - b0);
    const double Gam = 0.5 * (dir * (bl - b0) - M_PI);
    const double centre = frame_u ? (double)frame_u[a] : 0.5 * (U - 1);
    const double dn = frame_dist ? (double)frame_dist[a] : (double)sid[a];
    const double uc = ((double)u - centre) * (double)px;
    const double gam = dir * atan(uc / dn);
    double w = 0.0;
    if (beta >= 0.0 && beta < 2.0 * (Gam - gam)) {
        const double sw = sin(0.25 * M_PI * beta / (Gam - gam));
        w = sw * sw;
    } else if (beta >= 0.0 && beta <= M_PI - 2.0 * gam) {
        w = 1.0;
    } else if (beta > M_PI - 2.0 * gam && beta <= M_PI + 2.0 * Gam) {
        const double sw = sin(0.25 * M_PI * (M_PI + 2.0 * Gam - beta) / (Gam + gam));
        w = sw * sw;
    }
    out[i] = (float)w;
}

int fdk_parker_weights(const float* angles, const float* sid, const float* frame_dist,
                       const float* frame_u, int A, int U, float pixel_size, float* weights,
                       cudaStream_t s) {
    DGC_TRACE("parker_weights", s);
    const long long n = (long long)A * U;
    parker_weights_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        angles, sid, frame_dist, frame_u, A, U, pixel_size, weights);
    DGC_LAUNCH_CHECK("parker_weights");
    return DGC_OK;
}

int fdk_launch_filter(const FdkArgs& p, cudaStream_t s) {
    DGC_TRACE("fdk_filter_kernel", s);
    if (p.A > 65535) {
        set_error("fdk filter: more than 65535 views per launch");
        return DGC_ERR_UNSUPPORTED;
    }
    const dim3 grid(ceil_div(p.V, FBN), ceil_div(p.U, FBM), p.A);
    fdk_filter_kernel<false><<<grid, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fdk_filter_kernel");
    return DGC_OK;
}

long long fdk_filter_tiles(int U, int V) { return (long long)ceil_div(V, FBN) * ceil_div(U, FBM); }

int fdk_launch_filter_adjoint(const FdkArgs& p, cudaStream_t s) {
    DGC_TRACE("fdk_filter_adjoint_kernel", s);
    if (p.A > 65535) {
        set_error("fdk filter: more than 65535 views per launch");
        return DGC_ERR_UNSUPPORTED;
    }
    const dim3 grid(ceil_div(p.V, FBN), ceil_div(p.U, FBM), p.A);
    if (p.frame_grads)
        fdk_filter_kernel<true, true><<<grid, 256, 0, s>>>(p);
    else
        fdk_filter_kernel<true, false><<<grid, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fdk_filter_adjoint_kernel");
    return DGC_OK;
}

int fdk_reduce_distance_grads(const double* partials, int A, long long tiles, const FdkArgs& p,
                              const FdkGrads& g, cudaStream_t s) {
    DGC_TRACE("fdk_distance_grads", s);
    fdk_distance_grads_kernel<<<A, 32, 0, s>>>(partials, tiles, p, g);
    DGC_LAUNCH_CHECK("fdk_distance_grads");
    return DGC_OK;
}

int fdk_upload_taps(int U, float px, float alpha, float* dst, cudaStream_t s) {
    std::vector<double> h;
    int rc = fdk_taps_host(U, (double)px, (double)alpha, h);
    if (rc != DGC_OK) return rc;
    // Pinned staging buffer owned per thread; the copy is made stream-ordered
    // and the host waits for it before the buffer is reused.
    static thread_local float* staging = nullptr;
    static thread_local size_t staging_n = 0;
    static thread_local cudaEvent_t done = nullptr;
    if (staging_n < (size_t)U) {
        if (staging) {
            if (done) cudaEventSynchronize(done);
            cudaFreeHost(staging);
            staging = nullptr;
            staging_n = 0;
        }
        DGC_CUDA(cudaMallocHost(&staging, sizeof(float) * (size_t)U));
        staging_n = (size_t)U;
    }
    if (!done) DGC_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    DGC_CUDA(cudaEventSynchronize(done));
    for (int i = 0; i < U; ++i) staging[i] = (float)h[i];
    DGC_CUDA(cudaMemcpyAsync(dst, staging, sizeof(float) * (size_t)U, cudaMemcpyHostToDevice, s));
    DGC_CUDA(cudaEventRecord(done, s));
    return DGC_OK;
}

}  // namespace dgc

// ---------------------------------------------------------------------------
// Allocation-free variant (dgc_fdk_filter_noalloc, see include/dgc.h)
// ---------------------------------------------------------------------------

// Scratch of the allocation-free entry point: the filter's spectrum H[k],
// k in [0, P/2] (P/2 <= DGC_FDK_NOALLOC_MAX_U for U <= DGC_FDK_NOALLOC_MAX_U),
// and its taps h[m], m in [0, U).  98 KiB held by every GPU that loads the
// library.  Host code must not pass this name to a kernel (on the host it is
// only a stand-in symbol); its device address comes from cudaGetSymbolAddress.
struct NoallocScratch {
    double spectrum[DGC_FDK_NOALLOC_MAX_U + 1];
    float taps[DGC_FDK_NOALLOC_MAX_U];
};
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

namespace dgc {
namespace {

// fdk_taps_host's first sum on the device, one warp per bin k (lanes split
// the odd n, then a shuffle tree): H[k] = R[k] * hann[k].  cospi's argument
// 2j/P is exact because P is a power of two.
__global__ void noalloc_spectrum_kernel(double* H, int P, double px, double alpha) {
    const int half = P / 2;
    const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k > half) return;
    const unsigned mask = (unsigned)P - 1u;
    double R = 0.0;
    for (int n = 1 + 2 * lane; n <= half; n += 64) {
        const double pn = M_PI * (double)n * px;
        const double weight = (n == half) ? 1.0 : 2.0;
        const unsigned j = ((unsigned)k * (unsigned)n) & mask;
        R += weight * (-1.0 / (pn * pn)) * cospi(2.0 * (double)j / (double)P);
    }
    for (int o = 16; o > 0; o >>= 1) R += __shfl_xor_sync(0xffffffffu, R, o);
    if (lane == 0) {
        R += 1.0 / (4.0 * px * px);
        const double f = (k == half) ? -0.5 : (double)k / (double)P;
        const double hann = fabs(f) <= alpha * 0.5 ? 0.5 + 0.5 * cospi(2.0 * f / alpha) : 0.0;
        H[k] = R * hann;
    }
}

// fdk_taps_host's second sum, one warp per tap m:
// h[m] = (H[0] + 2 sum_{0<k<P/2} H[k] cos(2 pi k m / P) + H[P/2] cos(pi m)) / P.
__global__ void noalloc_taps_kernel(const double* H, int P, int U, float* taps) {
    const int half = P / 2;
    const int m = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (m >= U) return;
    const unsigned mask = (unsigned)P - 1u;
    double acc = 0.0;
    for (int k = 1 + lane; k < half; k += 32) {
        const unsigned j = ((unsigned)k * (unsigned)m) & mask;
        acc += 2.0 * H[k] * cospi(2.0 * (double)j / (double)P);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        acc += H[0] + H[half] * ((m & 1) ? -1.0 : 1.0);
        taps[m] = (float)(acc / (double)P);
    }
}

std::mutex g_noalloc_mu;
std::map<int, char*> g_noalloc_scratch_by_device;

// Device address of g_noalloc_scratch on the current device.  The first call
// on a device looks it up (loading the library's module there if needed) and
// caches it for the process; a cudaDeviceReset of that device invalidates the
// cached address.
int noalloc_scratch_address(char** out) {
    int dev = 0;
    DGC_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    auto it = g_noalloc_scratch_by_device.find(dev);
    if (it != g_noalloc_scratch_by_device.end()) {
        *out = it->second;
        return DGC_OK;
    }
    void* p = nullptr;
    DGC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_scratch_by_device[dev] = static_cast<char*>(p);
    *out = static_cast<char*>(p);
    return DGC_OK;
}

}  // namespace
}  // namespace dgc

extern "C" int dgc_fdk_filter_noalloc(const float* projections, int A, int U, int V,
                                      float pixel_size, const float* sod, const float* sid,
                                      float alpha, float* filtered, void* stream) {
    using namespace dgc;
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    DGC_REQUIRE(A > 0 && U > 0 && V > 0, "projections must have a nonempty [A, U, V] shape");
    DGC_REQUIRE(std::isfinite(pixel_size) && pixel_size > 0.0f,
                "pixel_size must be finite and positive");
    DGC_REQUIRE(std::isfinite(alpha) && alpha > 0.0f, "alpha must be finite and positive");
    DGC_REQUIRE(alpha <= 1.0f, "alpha must satisfy 0 < alpha <= 1");
    DGC_REQUIRE(projections && sod && sid && filtered, "pointers must be non-null");
    if (U > DGC_FDK_NOALLOC_MAX_U) {
        set_error("dgc_fdk_filter_noalloc: U = " + std::to_string(U) + " exceeds the " +
                  std::to_string(DGC_FDK_NOALLOC_MAX_U) +
                  "-tap static scratch; use dgc_fdk_filter with a workspace");
        return DGC_ERR_UNSUPPORTED;
    }
    char* scratch = nullptr;
    int rc = noalloc_scratch_address(&scratch);
    if (rc != DGC_OK) return rc;
    double* spectrum = reinterpret_cast<double*>(scratch + offsetof(NoallocScratch, spectrum));
    float* taps = reinterpret_cast<float*>(scratch + offsetof(NoallocScratch, taps));
    int bl = 0;
    for (int n = 2 * U - 1; n; n >>= 1) ++bl;
    const int P = 1 << bl;
    // The taps are written on the device, in stream order before the filter
    // reads them: the call reads no host memory after it returns and does not
    // wait for the stream.
    {
        DGC_TRACE("noalloc_spectrum_kernel", s);
        noalloc_spectrum_kernel<<<ceil_div((long long)(P / 2 + 1) * 32, 256), 256, 0, s>>>(
            spectrum, P, (double)pixel_size, (double)alpha);
        DGC_LAUNCH_CHECK("noalloc_spectrum_kernel");
    }
    {
        DGC_TRACE("noalloc_taps_kernel", s);
        noalloc_taps_kernel<<<ceil_div((long long)U * 32, 256), 256, 0, s>>>(spectrum, P, U, taps);
        DGC_LAUNCH_CHECK("noalloc_taps_kernel");
    }
    FdkArgs f{projections, sod, sid, taps, filtered, A, U, V, pixel_size};
    return fdk_launch_filter(f, s);
}

