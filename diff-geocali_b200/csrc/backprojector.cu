// backprojector.cu -- voxel-driven, FDK-weighted cone-beam backprojector and
// its hand-written backward, for sm_100a.
//
// Semantics follow the reference kernels of TomSHINING/diff-geoCali,
// csrc/src_cbct_backprojector_cuda.cu:
//   forward   15-98  : vol[z,y,x] = sum_a mask * ((sod+ds_n)/q)^2 * bilerp(P_a, u_idx, v_idx)
//   backward 101-295 : grad_proj (bilinear scatter) + d/d(sid, sod, beta, u0, v0, src_xyz)
//
// B200 design (not the reference's):
//   * A warp owns one (x, y) voxel column; its lanes walk Z (lane + 32k).  For a
//     fixed column and view, u_idx, the magnification t and the FDK weight do
//     not depend on z, and the lanes read one detector row pair at nearby V
//     positions (coalesced).
//   * Per-view trig and source terms are tabulated once per call; within a
//     warp, lane j evaluates the column geometry of view a0+j and the warp
//     broadcasts it with shuffles, so no lane recomputes it.
//   * Projections are re-laid out as quads PQ[a][u][v] = float4(P[u][v],
//     P[u][v+1], P[u+1][v], P[u+1][v+1]): one 16-byte load per voxel-view.
//   * Outputs go through a shared-memory transpose so the volume is written
//     along X (coalesced).
//   * The backward sums the per-voxel terms over Z in four accumulators and
//     applies the (column, view) chain-rule coefficients once per warp; the
//     eight per-view gradients are reduced in FP64 in a fixed order.
#include <mutex>

#include "common.cuh"
#include "backprojector.cuh"

namespace dgc {

// ---------------------------------------------------------------------------
// Per-view table and projection re-layout
// ---------------------------------------------------------------------------

__global__ void bp_view_table_kernel(Geometry g, int A, ViewRow* __restrict__ vt) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A) return;
    const float beta = g.angles[a];
    const float c = cosf(beta);
    const float s = sinf(beta);
    ViewRow r;
    r.c = c;
    r.s = s;
    // World-coordinate source offset in the rotating system (bp.cu:53-56).
    r.ds_u = g.src_x[a] * c + g.src_y[a] * s;
    r.ds_n = -g.src_x[a] * s + g.src_y[a] * c;
    r.ds_v = g.src_z[a];
    r.sod = g.sod[a];
    r.sid = g.sid[a];
    r.u0 = g.det_u0[a];
    r.v0 = g.det_v0[a];
    r.pad0 = r.pad1 = r.pad2 = 0.0f;
    vt[a] = r;
}

int bp_view_table(const Geometry& g, int A, ViewRow* vt, cudaStream_t s) {
    DGC_TRACE("bp_view_table", s);
    bp_view_table_kernel<<<ceil_div(A, 128), 128, 0, s>>>(g, A, vt);
    DGC_LAUNCH_CHECK("bp_view_table");
    return DGC_OK;
}

__global__ void build_proj_quads_kernel(const float* __restrict__ P, int A, int U, int V,
                                        float4* __restrict__ PQ) {
    const int QU = U - 1, QV = V - 1;
    const long long total = (long long)A * QU * QV;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(i % QV);
        const long long r = i / QV;
        const int u = (int)(r % QU);
        const int a = (int)(r / QU);
        const float* row = P + ((long long)a * U + u) * V + v;
        PQ[i] = make_float4(__ldg(row), __ldg(row + 1), __ldg(row + V), __ldg(row + V + 1));
    }
}

int build_proj_quads(const float* P, int A, int U, int V, float4* PQ, cudaStream_t s) {
    DGC_TRACE("build_proj_quads", s);
    const long long total = (long long)A * (U - 1) * (V - 1);
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    build_proj_quads_kernel<<<blocks, 256, 0, s>>>(P, A, U, V, PQ);
    DGC_LAUNCH_CHECK("build_proj_quads");
    return DGC_OK;
}

// ---------------------------------------------------------------------------
// Column geometry of one (x, y, view) (bp.cu:48-79)
// ---------------------------------------------------------------------------

struct ColumnView {
    bool valid;   // q, sid+ds_n > 1e-6 and 0 <= u_idx < U-1
    int row;      // quad-row index (a*(U-1) + u0)*(V-1)
    float t;      // magnification (sid+ds_n)/q
    float w;      // ((sod+ds_n)/q)^2
    float fu;     // u_idx - u0
    float ds_v;
    float v0;
};

template <bool PIXDIV>
__device__ __forceinline__ ColumnView column_view(const ViewRow& r, int a, float vx, float vy,
                                                  const BpArgs& p) {
    ColumnView cv;
    cv.valid = false;
    cv.row = 0;
    cv.t = cv.w = cv.fu = cv.ds_v = cv.v0 = 0.0f;
    const float px = vx * r.c + vy * r.s;
    const float py = -vx * r.s + vy * r.c;
    const float denom = r.sod + r.ds_n - py;
    const float sdn = r.sid + r.ds_n;
    if (!(denom > 1e-6f && sdn > 1e-6f)) return cv;
    const float t = sdn / denom;
    const float u_phys = r.ds_u + t * (px - r.ds_u);
    const float sw = (r.sod + r.ds_n) / denom;
    const float u_idx = PIXDIV ? u_phys / p.pixel_size + r.u0 : fmaf(u_phys, p.inv_pixel, r.u0);
    if (!(u_idx >= 0.0f && u_idx < (p.U - 1.0f))) return cv;
    const int ui = (int)floorf(u_idx);
    cv.valid = true;
    cv.row = (a * (p.U - 1) + ui) * (p.V - 1);
    cv.t = t;
    cv.w = sw * sw;
    cv.fu = u_idx - ui;
    cv.ds_v = r.ds_v;
    cv.v0 = r.v0;
    return cv;
}

// ---------------------------------------------------------------------------
// Forward (backprojection) kernel
// ---------------------------------------------------------------------------

// A CTA owns a cta_x x cta_y patch of (x, y) columns, one warp per column
// (at most kBpMaxWarps warps), and 32*KZ voxels of each along z.
template <int KZ, bool PIXDIV, bool FDK>
__global__ void __launch_bounds__(32 * kBpMaxWarps) bp_forward_kernel(BpArgs p) {
    __shared__ float s_out[32 * KZ][kBpMaxWarps + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cx = p.cta_x, cy = p.cta_y, nw = cx * cy;
    const int tiles_x = (p.W + cx - 1) / cx;
    const int ty = blockIdx.x / tiles_x;
    const int xb = (blockIdx.x - ty * tiles_x) * cx, yb = ty * cy;
    const int x = xb + warp % cx, y = yb + warp / cx;
    const int zbase = blockIdx.y * 32 * KZ;
    const unsigned FULL = 0xffffffffu;

    float acc[KZ];
    float pz[KZ];
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        acc[k] = 0.0f;
        const int z = zbase + lane + 32 * k;
        pz[k] = (z - p.D * 0.5f) * p.voxel_size + p.off_z;
    }
    if (x < p.W && y < p.H) {
        const float vx = (x - p.W * 0.5f) * p.voxel_size + p.off_x;
        const float vy = (y - p.H * 0.5f) * p.voxel_size + p.off_y;
        const float vlim = p.V - 1.0f;
        const int zlimit = p.D - zbase - lane;  // k valid while 32k < zlimit
        for (int a0 = 0; a0 < p.A; a0 += 32) {
            ColumnView mine;
            mine.valid = false;
            if (a0 + lane < p.A) mine = column_view<PIXDIV>(p.vt[a0 + lane], a0 + lane, vx, vy, p);
            const unsigned valid_mask = __ballot_sync(FULL, mine.valid);
            const int nv = min(32, p.A - a0);
            for (int j = 0; j < nv; ++j) {
                if (!((valid_mask >> j) & 1u)) continue;
                const float t = __shfl_sync(FULL, mine.t, j);
                const float dsv = __shfl_sync(FULL, mine.ds_v, j);
                const float v0 = __shfl_sync(FULL, mine.v0, j);
                const float w = __shfl_sync(FULL, mine.w, j);
                const float fu = __shfl_sync(FULL, mine.fu, j);
                const int row = __shfl_sync(FULL, mine.row, j);
                const float4* __restrict__ rq = p.pquads + row;
#pragma unroll
                for (int k = 0; k < KZ; ++k) {
                    const float v_phys = dsv + t * (pz[k] - dsv);
                    const float v_idx =
                        PIXDIV ? v_phys / p.pixel_size + v0 : fmaf(v_phys, p.inv_pixel, v0);
                    if (32 * k < zlimit && v_idx >= 0.0f && v_idx < vlim) {
                        const FloorSplit fs = floor_split(v_idx);
                        const float4 q = __ldg(rq + (int)(fs.biased - kFloorMagicBits));
                        const float interp =
                            lerpf(lerpf(q.x, q.y, fs.frac), lerpf(q.z, q.w, fs.frac), fu);
                        acc[k] = fmaf(w, interp, acc[k]);
                    }
                }
            }
        }
    }
    // Transpose through shared memory; write rows along X.
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        float val = acc[k];
        if (FDK) {
            val *= p.out_scale;
            if (p.clamp) val = val < 0.0f ? 0.0f : val;  // clamp_min(0); NaN propagates
        }
        s_out[lane + 32 * k][warp] = val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * KZ * nw; i += 32 * nw) {
        const int zl = i / nw, w = i - zl * nw;
        const int z = zbase + zl, xx = xb + w % cx, yy = yb + w / cx;
        if (z < p.D && xx < p.W && yy < p.H)
            p.volume[((long long)z * p.H + yy) * p.W + xx] = s_out[zl][w];
    }
}

// ---------------------------------------------------------------------------
// Backward kernel
// ---------------------------------------------------------------------------

// GP: projection gradient 0 = not computed (p.grad_projections null), 1 = four
// float reductions per voxel-view into grad_projections.
template <int KZ, int GP>
__global__ void __launch_bounds__(256) bp_backward_kernel(BpArgs p) {
    __shared__ double s_terms[8][32][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cols_x = (p.W + 7) >> 3;
    const int y = blockIdx.x / cols_x;
    const int x = (blockIdx.x - y * cols_x) * 8 + warp;
    const int zbase = blockIdx.y * 32 * KZ;
    const long long block_id = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    const long long nblocks = (long long)gridDim.x * gridDim.y;
    const bool col_ok = x < p.W;
    const float vx = (x - p.W * 0.5f) * p.voxel_size + p.off_x;
    const float vy = (y - p.H * 0.5f) * p.voxel_size + p.off_y;
    const float vlim = p.V - 1.0f;

    float gval[KZ], pz[KZ];
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        const int z = zbase + lane + 32 * k;
        pz[k] = (z - p.D * 0.5f) * p.voxel_size + p.off_z;
        gval[k] = (col_ok && z < p.D) ? p.grad_volume[((long long)z * p.H + y) * p.W + x] : 0.0f;
    }
    const int zlimit = p.D - zbase - lane;

    for (int a0 = 0; a0 < p.A; a0 += 32) {
        const int nv = min(32, p.A - a0);
        for (int j = 0; j < nv; ++j) {
            const int a = a0 + j;
            const ViewRow r = p.vt[a];
            float terms[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            // column geometry (backward form of bp.cu:139-174: u/v idx use 1/pixel)
            const float px = vx * r.c + vy * r.s;
            const float py = -vx * r.s + vy * r.c;
            const float denom = r.sod + r.ds_n - py;
            const float sdn = r.sid + r.ds_n;
            bool ok = col_ok && denom > 1e-6f && sdn > 1e-6f;
            float inv_q = 0.f, t = 0.f, du = 0.f, m = 0.f, w = 0.f, fu = 0.f;
            int ui = 0;
            if (ok) {
                inv_q = 1.0f / denom;
                t = sdn * inv_q;
                du = px - r.ds_u;
                const float u_phys = r.ds_u + t * du;
                m = r.sod + r.ds_n;
                w = m * m * (inv_q * inv_q);
                const float u_idx = u_phys * p.inv_pixel + r.u0;
                ok = u_idx >= 0.0f && u_idx < (p.U - 1.0f);
                if (ok) {
                    ui = (int)floorf(u_idx);
                    fu = u_idx - ui;
                }
            }
            if (ok) {  // warp-uniform
                float s_iu = 0.f, s_iv = 0.f, s_ivdv = 0.f, s_int = 0.f;
                const float4* __restrict__ rq = p.pquads + (a * (p.U - 1) + ui) * (p.V - 1);
                float* __restrict__ gp = GP ? p.grad_projections + ((long long)a * p.U + ui) * p.V
                                            : nullptr;
#pragma unroll
                for (int k = 0; k < KZ; ++k) {
                    const float dv = pz[k] - r.ds_v;
                    const float v_phys = r.ds_v + t * dv;
                    const float v_idx = v_phys * p.inv_pixel + r.v0;
                    if (32 * k < zlimit && v_idx >= 0.0f && v_idx < vlim) {
                        const FloorSplit fs = floor_split(v_idx);
                        const int vi = (int)(fs.biased - kFloorMagicBits);
                        const float fv = fs.frac;
                        const float4 q = __ldg(rq + vi);
                        const float interp = lerpf(lerpf(q.x, q.y, fv), lerpf(q.z, q.w, fv), fu);
                        const float iu = lerpf(q.z - q.x, q.w - q.y, fv);
                        const float iv = lerpf(q.y - q.x, q.w - q.z, fu);
                        const float g = gval[k];
                        s_iu = fmaf(g, iu, s_iu);
                        s_iv = fmaf(g, iv, s_iv);
                        s_ivdv = fmaf(g * iv, dv, s_ivdv);
                        s_int = fmaf(g, interp, s_int);
                        if (GP) {
                            const float gb = g * w;
                            const float g0 = gb * (1.0f - fu), g1 = gb * fu;
                            red_add_global(gp + vi, g0 * (1.0f - fv));
                            red_add_global(gp + p.V + vi, g1 * (1.0f - fv));
                            red_add_global(gp + vi + 1, g0 * fv);
                            red_add_global(gp + p.V + vi + 1, g1 * fv);
                        }
                    }
                }
                s_iu = warp_sum(s_iu);
                s_iv = warp_sum(s_iv);
                s_ivdv = warp_sum(s_ivdv);
                s_int = warp_sum(s_int);
                if (lane == 0) {
                    // Chain-rule coefficients of bp.cu:213-292, applied to the
                    // Z sums: sum g*(Iu*dU + Iv*dV) = dU*s_iu + dt*s_ivdv, etc.
                    const float inv_q2 = inv_q * inv_q, inv_q3 = inv_q2 * inv_q;
                    const float m2 = m * m;
                    const float ip = p.inv_pixel;
                    const float b_sid = du * s_iu + s_ivdv;
                    terms[1] = w * inv_q * ip * b_sid;
                    const float dt_sod = -sdn * inv_q2;
                    const float dw_sod = 2.0f * m * inv_q2 - 2.0f * m2 * inv_q3;
                    terms[2] = dw_sod * s_int + w * ip * dt_sod * b_sid;
                    const float dsu_b = r.ds_n, dsn_b = -r.ds_u, dq_b = du;
                    const float dt_b = (dsn_b * denom - sdn * dq_b) * inv_q2;
                    const float du_b = (1.0f - t) * dsu_b + t * py + du * dt_b;
                    const float dw_b = 2.0f * m * inv_q2 * dsn_b - 2.0f * m2 * inv_q3 * dq_b;
                    terms[0] = dw_b * s_int + w * ip * (du_b * s_iu + dt_b * s_ivdv);
                    terms[3] = w * s_iu;
                    terms[4] = w * s_iv;
                    const float dsu_x = r.c, dsn_x = -r.s;
                    const float dt_x = dsn_x * (denom - sdn) * inv_q2;
                    const float du_x = (1.0f - t) * dsu_x + du * dt_x;
                    const float dw_x = 2.0f * m * inv_q2 * dsn_x - 2.0f * m2 * inv_q3 * dsn_x;
                    terms[5] = dw_x * s_int + w * ip * (du_x * s_iu + dt_x * s_ivdv);
                    const float dsu_y = r.s, dsn_y = r.c;
                    const float dt_y = dsn_y * (denom - sdn) * inv_q2;
                    const float du_y = (1.0f - t) * dsu_y + du * dt_y;
                    const float dw_y = 2.0f * m * inv_q2 * dsn_y - 2.0f * m2 * inv_q3 * dsn_y;
                    terms[6] = dw_y * s_int + w * ip * (du_y * s_iu + dt_y * s_ivdv);
                    terms[7] = w * (1.0f - t) * ip * s_iv;
                }
            }
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < 8; ++k) s_terms[warp][j][k] = (double)terms[k];
            }
        }
        __syncthreads();
        {
            const int j = threadIdx.x >> 3, k = threadIdx.x & 7;
            if (j < nv) {
                double acc = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) acc += s_terms[w][j][k];
                p.partials[((long long)(a0 + j) * 8 + k) * nblocks + block_id] = acc;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) bp_reduce_partials_kernel(const double* __restrict__ partials,
                                                                 long long nblocks, GeometryGrad out) {
    const int a = blockIdx.x;
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double* src = partials + ((long long)a * 8 + k) * nblocks;
    double acc = 0.0;
    for (long long i = lane; i < nblocks; i += 32) acc += src[i];
    acc = warp_sum(acc);
    if (lane == 0) out.g[k][a] = (float)acc;
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

// Z values per lane (a warp covers 32*KZ voxels of a column, a CTA 8 columns).
// Fewer Z per warp keep the projection rows a CTA reads per view short, so
// they stay in L1; more amortise the per-(column, view) geometry.  Measured
// (sid 1000, sod 600; 256^3 / 360 x 384^2, 128^3 / 180 x 256^2, 512^3 / 90 x
// 512^2), forward KZ = 1 / 2 / 4 / 8: 9.07 / 8.18 / 11.6 / 14.1 ms,
// 0.46 / 0.36 / 0.52 / 0.52 ms, 17.0 / 13.7 / 14.5 / 15.5 ms; backward
// without the projection gradient: 45.9 / 28.7 / 21.3 / 28.2 ms,
// 2.38 / 1.43 / 1.04 / 1.34 ms, 96.0 / 56.2 / 37.1 / 45.6 ms (with it
// 36.1-36.9 ms at KZ 2-4 for 256^3, 62.0 ms at KZ 4 for 512^3).
// Tile rules registered by the autotuner (dgc_bp_add_tile_rule): the first
// rule with D <= d_max and A <= a_max applies; a zero field keeps the
// built-in choice.
namespace {
struct BpTileRule {
    int d_max, a_max, kz_forward, kz_backward, cta_x, cta_y;
};
std::mutex g_rule_mutex;
BpTileRule g_rules[kBpMaxTileRules];
int g_rule_count = 0;

bool bp_rule(int D, int A, BpTileRule& out) {
    std::lock_guard<std::mutex> lock(g_rule_mutex);
    for (int i = 0; i < g_rule_count; ++i)
        if (D <= g_rules[i].d_max && A <= g_rules[i].a_max) {
            out = g_rules[i];
            return true;
        }
    return false;
}

bool valid_kz(int k) { return k == 0 || k == 1 || k == 2 || k == 4 || k == 8; }
}  // namespace

int bp_add_tile_rule(int d_max, int a_max, int kz_forward, int kz_backward, int cta_x, int cta_y) {
    if (d_max < 1 || a_max < 1 || !valid_kz(kz_forward) || !valid_kz(kz_backward)) return -1;
    const bool cta_default = cta_x == 0 && cta_y == 0;
    if (!cta_default && (cta_x < 1 || cta_y < 1 || cta_x * cta_y > kBpMaxWarps)) return -1;
    std::lock_guard<std::mutex> lock(g_rule_mutex);
    if (g_rule_count >= kBpMaxTileRules) return -2;
    g_rules[g_rule_count++] = BpTileRule{d_max, a_max, kz_forward, kz_backward, cta_x, cta_y};
    return 0;
}

void bp_clear_tile_rules() {
    std::lock_guard<std::mutex> lock(g_rule_mutex);
    g_rule_count = 0;
}

int bp_kz_forward(int D, int A) {
    BpTileRule r;
    if (bp_rule(D, A, r) && r.kz_forward) return r.kz_forward;
    return D <= 32 ? 1 : 2;
}

int bp_kz_backward(int D, int A) {
    BpTileRule r;
    if (bp_rule(D, A, r) && r.kz_backward) return r.kz_backward;
    return D <= 32 ? 1 : D <= 64 ? 2 : 4;
}

// Column patch of a forward CTA (cx*cy <= kBpMaxWarps); 8 x 1 built in.
void bp_forward_cta(int D, int A, int& cx, int& cy) {
    BpTileRule r;
    if (bp_rule(D, A, r) && r.cta_x) {
        cx = r.cta_x;
        cy = r.cta_y;
        return;
    }
    cx = 8;
    cy = 1;
}

void bp_grid(int D, int H, int W, int kz, unsigned& gx, unsigned& gy) {
    gx = (unsigned)(((W + 7) / 8) * (long long)H);
    gy = (unsigned)ceil_div(D, 32 * kz);
}

long long bp_backward_blocks(int D, int H, int W, int kz) {
    unsigned gx, gy;
    bp_grid(D, H, W, kz, gx, gy);
    return (long long)gx * gy;
}

namespace {
template <int KZ>
int launch_bp_forward_kz(const BpArgs& p, bool pixdiv, bool fdk, dim3 grid, cudaStream_t s) {
    const unsigned threads = 32u * (unsigned)(p.cta_x * p.cta_y);
    if (fdk) {
        if (pixdiv) bp_forward_kernel<KZ, true, true><<<grid, threads, 0, s>>>(p);
        else bp_forward_kernel<KZ, false, true><<<grid, threads, 0, s>>>(p);
    } else {
        if (pixdiv) bp_forward_kernel<KZ, true, false><<<grid, threads, 0, s>>>(p);
        else bp_forward_kernel<KZ, false, false><<<grid, threads, 0, s>>>(p);
    }
    DGC_LAUNCH_CHECK("bp_forward_kernel");
    return DGC_OK;
}

template <int KZ>
int launch_bp_backward_kz(const BpArgs& p, int gp, dim3 grid, cudaStream_t s) {
    if (gp) bp_backward_kernel<KZ, 1><<<grid, 256, 0, s>>>(p);
    else bp_backward_kernel<KZ, 0><<<grid, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("bp_backward_kernel");
    return DGC_OK;
}
}  // namespace

int bp_launch_forward(const BpArgs& args, bool fdk, cudaStream_t s) {
    DGC_TRACE(fdk ? "bp_forward_kernel<fdk>" : "bp_forward_kernel", s);
    BpArgs p = args;
    bp_forward_cta(p.D, p.A, p.cta_x, p.cta_y);
    const bool pixdiv = !is_pow2_float(p.pixel_size);
    const int kz = bp_kz_forward(p.D, p.A);
    const dim3 grid((unsigned)(ceil_div(p.W, p.cta_x) * (long long)ceil_div(p.H, p.cta_y)),
                    (unsigned)ceil_div(p.D, 32 * kz));
    switch (kz) {
        case 1: return launch_bp_forward_kz<1>(p, pixdiv, fdk, grid, s);
        case 2: return launch_bp_forward_kz<2>(p, pixdiv, fdk, grid, s);
        case 4: return launch_bp_forward_kz<4>(p, pixdiv, fdk, grid, s);
        default: return launch_bp_forward_kz<8>(p, pixdiv, fdk, grid, s);
    }
}

int bp_launch_backward(const BpArgs& p, cudaStream_t s) {
    DGC_TRACE("bp_backward_kernel", s);
    // the Z blocking the caller sized the partials for (a rule added by another
    // thread in between must not change the grid)
    const int kz = p.kz_backward ? p.kz_backward : bp_kz_backward(p.D, p.A);
    unsigned gx, gy;
    bp_grid(p.D, p.H, p.W, kz, gx, gy);
    const dim3 grid(gx, gy);
    const int gp = p.grad_projections ? 1 : 0;
    switch (kz) {
        case 1: return launch_bp_backward_kz<1>(p, gp, grid, s);
        case 2: return launch_bp_backward_kz<2>(p, gp, grid, s);
        case 4: return launch_bp_backward_kz<4>(p, gp, grid, s);
        default: return launch_bp_backward_kz<8>(p, gp, grid, s);
    }
}

__global__ void clamp_volume_kernel(float* __restrict__ v, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float x = v[i];
        v[i] = x < 0.0f ? 0.0f : x;  // as the FDK epilogue: NaN propagates
    }
}

int bp_clamp_volume(float* volume, long long n, cudaStream_t s) {
    DGC_TRACE("clamp_volume", s);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    clamp_volume_kernel<<<blocks, 256, 0, s>>>(volume, n);
    DGC_LAUNCH_CHECK("clamp_volume");
    return DGC_OK;
}

int bp_reduce_partials(const double* partials, int A, long long nblocks, const GeometryGrad& out,
                       cudaStream_t s) {
    DGC_TRACE("bp_reduce_partials", s);
    bp_reduce_partials_kernel<<<A, 256, 0, s>>>(partials, nblocks, out);
    DGC_LAUNCH_CHECK("bp_reduce_partials");
    return DGC_OK;
}

}  // namespace dgc
