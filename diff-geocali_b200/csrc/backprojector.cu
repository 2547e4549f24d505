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
//     P[u+1][v], P[u][v+1], P[u+1][v+1]) -- two column pairs, so the lerp
//     along v runs as one packed f32x2 lerp over rows u and u+1: one 16-byte
//     load per voxel-view.
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
        PQ[i] = make_float4(__ldg(row), __ldg(row + V), __ldg(row + 1), __ldg(row + V + 1));
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
// Block order
// ---------------------------------------------------------------------------

// Tile (tx, ty) and z block of a CTA from its linear index.  Every CTA loops
// over all views, so the projection data a CTA reads per view is re-read from
// DRAM by each wave of CTAs unless the CTAs in flight share it: they must
// cover a compact region of the volume, whose projections are small patches
// of each view (a strip of rows along the whole volume width projects onto
// whole detector rows).  Tiles are therefore taken z block by z block and,
// inside a z block, in super-tiles of sx x sy tiles (about 64 x 64 voxels,
// one wave of CTAs) ordered row by row; edge super-tiles are narrower.
struct BpTile {
    int tx, ty, zb;
};

__device__ __forceinline__ BpTile bp_tile(long long linear, int tiles_x, int tiles_y, int sx,
                                          int sy) {
    const long long layer = (long long)tiles_x * tiles_y;
    BpTile t;
    t.zb = (int)(linear / layer);
    const long long r = linear - (long long)t.zb * layer;
    const long long band_tiles = (long long)sy * tiles_x;
    const int band = (int)(r / band_tiles);
    const long long rb = r - band * band_tiles;
    const int rows = min(sy, tiles_y - band * sy);
    const int col = (int)(rb / ((long long)sx * rows));
    const int rc = (int)(rb - (long long)col * sx * rows);
    const int cols = min(sx, tiles_x - col * sx);
    t.ty = band * sy + rc / cols;
    t.tx = col * sx + rc % cols;
    return t;
}

__host__ __device__ __forceinline__ int bp_super(int cta) { return cta >= 64 ? 1 : 64 / cta; }

// ---------------------------------------------------------------------------
// Forward (backprojection) kernel
// ---------------------------------------------------------------------------

// A CTA owns a cta_x x cta_y patch of (x, y) columns, one warp per column
// (at most kBpMaxWarps warps), and 32*KZ voxels of each along z.
//
// Register caps by z depth (in place of launch bounds, which cannot express
// "five 256-thread CTAs per SM"): at KZ = 2 the compiler's own choice (49
// registers) leaves four CTAs per SM and runs 1.5x slower than 48 registers
// and five CTAs.  Any CTA of up to kBpMaxWarps warps fits under each cap.
template <int KZ, bool PIXDIV, bool FDK>
__global__ void __maxnreg__(KZ == 1 ? 40 : KZ == 2 ? 48 : KZ == 4 ? 64 : 96) bp_forward_kernel(BpArgs p) {
    __shared__ float s_out[32 * KZ][kBpMaxWarps + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cx = p.cta_x, cy = p.cta_y, nw = cx * cy;
    const int tiles_x = (p.W + cx - 1) / cx, tiles_y = (p.H + cy - 1) / cy;
    const BpTile tile = bp_tile((long long)blockIdx.y * gridDim.x + blockIdx.x, tiles_x, tiles_y,
                                bp_super(cx), bp_super(cy));
    const int xb = tile.tx * cx, yb = tile.ty * cy;
    const int x = xb + warp % cx, y = yb + warp / cx;
    const int zbase = tile.zb * 32 * KZ;
    const unsigned FULL = 0xffffffffu;

    // FP32 sums of up to 8 views, added into FP64 totals: the FDK terms of a
    // voxel cancel over the views (filtered projections change sign), and a
    // running FP32 sum over hundreds of views loses 1e-5 to 1e-4 of the
    // result to that cancellation
    double acc[KZ];
    float part[KZ];
    float pz[KZ];
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        acc[k] = 0.0;
        part[k] = 0.0f;
        const int z = zbase + lane + 32 * k;
        pz[k] = (z - p.D * 0.5f) * p.voxel_size + p.off_z;
    }
    if (x < p.W && y < p.H) {
        const float vx = (x - p.W * 0.5f) * p.voxel_size + p.off_x;
        const float vy = (y - p.H * 0.5f) * p.voxel_size + p.off_y;
        const int zlimit = p.D - zbase - lane;  // k valid while 32k < zlimit
        // a tap is valid iff 0 <= v_idx < V-1, i.e. its floor (exact from the
        // magic-number split, which maps NaN, infinities and values beyond
        // 2^22 outside [0, V-2]) as an unsigned index is below V-1
        const uint32_t vcount = (uint32_t)max(p.V - 1, 0);
        f32x2 pz2[KZ / 2 > 0 ? KZ / 2 : 1];
#pragma unroll
        for (int k = 0; k + 1 < KZ; k += 2) pz2[k / 2] = pack2(pz[k], pz[k + 1]);
        const f32x2 ip2 = pack2(p.inv_pixel, p.inv_pixel);
        const f32x2 magic2 = pack2(kFloorMagic, kFloorMagic);
        for (int a0 = 0; a0 < p.A; a0 += 32) {
            ColumnView mine;
            mine.valid = false;
            if (a0 + lane < p.A) mine = column_view<PIXDIV>(p.vt[a0 + lane], a0 + lane, vx, vy, p);
            const unsigned valid_mask = __ballot_sync(FULL, mine.valid);
            const int nv = min(32, p.A - a0);
            // views in chunks of 8, each chunk's FP32 partial sums added into
            // the FP64 totals after it
            for (int jb = 0; jb < nv; jb += 8) {
                const int je = min(jb + 8, nv);
                for (int j = jb; j < je; ++j) {
                    if (!((valid_mask >> j) & 1u)) continue;
                    const float t = __shfl_sync(FULL, mine.t, j);
                    const float dsv = __shfl_sync(FULL, mine.ds_v, j);
                    const float v0 = __shfl_sync(FULL, mine.v0, j);
                    const float w = __shfl_sync(FULL, mine.w, j);
                    const float fu = __shfl_sync(FULL, mine.fu, j);
                    const int row = __shfl_sync(FULL, mine.row, j);
                    const ulonglong2* __restrict__ rq =
                        reinterpret_cast<const ulonglong2*>(p.pquads) + row;
                    // one tap: v_idx's floor split -> validity, column pair lerp
                    // along v (packed: rows u and u+1), then along u
                    auto tap = [&](int k, uint32_t biased, float fv) {
                        const uint32_t vi = biased - kFloorMagicBits;
                        if (32 * k < zlimit && vi < vcount) {
                            const ulonglong2 q = __ldg(rq + vi);
                            const float2 e = unpack2(lerp2(q.x, q.y, pack2(fv, fv)));
                            part[k] = fmaf(w, lerpf(e.x, e.y, fu), part[k]);
                        }
                    };
                    if constexpr (!PIXDIV && KZ % 2 == 0) {
                        const f32x2 t2 = pack2(t, t), d2 = pack2(dsv, dsv), o2 = pack2(v0, v0);
#pragma unroll
                        for (int k = 0; k < KZ; k += 2) {
                            const f32x2 vp = fma2(t2, sub2(pz2[k / 2], d2), d2);
                            const f32x2 vx2 = fma2(vp, ip2, o2);
                            const f32x2 f2 = add2_rd(vx2, magic2);
                            const float2 fr = unpack2(sub2(vx2, sub2(f2, magic2)));
                            const uint2 bits = unpack2_bits(f2);
                            tap(k, bits.x, fr.x);
                            tap(k + 1, bits.y, fr.y);
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < KZ; ++k) {
                            const float v_phys = dsv + t * (pz[k] - dsv);
                            const float v_idx =
                                PIXDIV ? v_phys / p.pixel_size + v0 : fmaf(v_phys, p.inv_pixel, v0);
                            const FloorSplit fs = floor_split(v_idx);
                            tap(k, fs.biased, fs.frac);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < KZ; ++k) {
                    acc[k] += (double)part[k];
                    part[k] = 0.0f;
                }
            }
        }
    }
    // Transpose through shared memory; write rows along X.
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        float val = FDK ? (float)(acc[k] * (double)p.out_scale) : (float)acc[k];
        if (FDK) {
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

// Column geometry of one (x, y, view) for the backward (bp.cu:139-174; the
// u/v indices use 1/pixel) and what the chain rule of bp.cu:213-292 needs.
struct ColumnGrad {
    bool ok;
    int ui;
    float t, w, fu, inv_q, du, m, sdn, denom, py;
    float ds_u, ds_n, ds_v, v0, c, s;
};

__device__ __forceinline__ ColumnGrad column_grad(const ViewRow& r, float vx, float vy, bool col_ok,
                                                  const BpArgs& p) {
    ColumnGrad g;
    g.c = r.c;
    g.s = r.s;
    g.ds_u = r.ds_u;
    g.ds_n = r.ds_n;
    g.ds_v = r.ds_v;
    g.v0 = r.v0;
    g.ui = 0;
    g.t = g.w = g.fu = g.inv_q = g.du = g.m = 0.f;
    const float px = vx * r.c + vy * r.s;
    g.py = -vx * r.s + vy * r.c;
    g.denom = r.sod + r.ds_n - g.py;
    g.sdn = r.sid + r.ds_n;
    g.ok = col_ok && g.denom > 1e-6f && g.sdn > 1e-6f;
    if (g.ok) {
        g.inv_q = 1.0f / g.denom;
        g.t = g.sdn * g.inv_q;
        g.du = px - r.ds_u;
        const float u_phys = r.ds_u + g.t * g.du;
        g.m = r.sod + r.ds_n;
        g.w = g.m * g.m * (g.inv_q * g.inv_q);
        const float u_idx = u_phys * p.inv_pixel + r.u0;
        g.ok = u_idx >= 0.0f && u_idx < (p.U - 1.0f);
        if (g.ok) {
            g.ui = (int)floorf(u_idx);
            g.fu = u_idx - g.ui;
        }
    }
    return g;
}

// The eight per-view geometry gradients of a (column, view) from its four Z
// sums (s_iu = sum g*Iu, s_iv = sum g*Iv, s_ivdv = sum g*Iv*dv, s_int = sum
// g*interp): the chain-rule coefficients of bp.cu:213-292 applied once.
__device__ __forceinline__ void column_terms(const ColumnGrad& g, float s_iu, float s_iv,
                                             float s_ivdv, float s_int, float ip,
                                             float (&terms)[8]) {
    const float inv_q2 = g.inv_q * g.inv_q, inv_q3 = inv_q2 * g.inv_q;
    const float m2 = g.m * g.m;
    const float b_sid = g.du * s_iu + s_ivdv;
    terms[1] = g.w * g.inv_q * ip * b_sid;
    const float dt_sod = -g.sdn * inv_q2;
    const float dw_sod = 2.0f * g.m * inv_q2 - 2.0f * m2 * inv_q3;
    terms[2] = dw_sod * s_int + g.w * ip * dt_sod * b_sid;
    const float dsu_b = g.ds_n, dsn_b = -g.ds_u, dq_b = g.du;
    const float dt_b = (dsn_b * g.denom - g.sdn * dq_b) * inv_q2;
    const float du_b = (1.0f - g.t) * dsu_b + g.t * g.py + g.du * dt_b;
    const float dw_b = 2.0f * g.m * inv_q2 * dsn_b - 2.0f * m2 * inv_q3 * dq_b;
    terms[0] = dw_b * s_int + g.w * ip * (du_b * s_iu + dt_b * s_ivdv);
    terms[3] = g.w * s_iu;
    terms[4] = g.w * s_iv;
    const float dsu_x = g.c, dsn_x = -g.s;
    const float dt_x = dsn_x * (g.denom - g.sdn) * inv_q2;
    const float du_x = (1.0f - g.t) * dsu_x + g.du * dt_x;
    const float dw_x = 2.0f * g.m * inv_q2 * dsn_x - 2.0f * m2 * inv_q3 * dsn_x;
    terms[5] = dw_x * s_int + g.w * ip * (du_x * s_iu + dt_x * s_ivdv);
    const float dsu_y = g.s, dsn_y = g.c;
    const float dt_y = dsn_y * (g.denom - g.sdn) * inv_q2;
    const float du_y = (1.0f - g.t) * dsu_y + g.du * dt_y;
    const float dw_y = 2.0f * g.m * inv_q2 * dsn_y - 2.0f * m2 * inv_q3 * dsn_y;
    terms[6] = dw_y * s_int + g.w * ip * (du_y * s_iu + dt_y * s_ivdv);
    terms[7] = g.w * (1.0f - g.t) * ip * s_iv;
}

// Sums of N (16 or 32) per-lane values over the warp, lane L receiving the
// sum of value L mod N: log2(N) butterfly steps, each halving the values a
// lane holds (N-1 shuffles for the N sums instead of 5 per sum), then the
// halves of the warp added.
template <int N>
__device__ __forceinline__ float warp_transpose_sum(float (&v)[N], int lane) {
    const unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int h = N / 2; h >= 1; h >>= 1) {
        const bool up = (lane & h) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const float send = up ? v[k] : v[k + h];
            const float keep = up ? v[k + h] : v[k];
            v[k] = keep + __shfl_xor_sync(FULL, send, h);
        }
    }
    float x = v[0];
#pragma unroll
    for (int o = N; o < 32; o <<= 1) x += __shfl_xor_sync(FULL, x, o);
    return x;
}

// Views whose four z-sums are reduced together (16 accumulators per lane).
constexpr int kBpGroup = 4;

// GP: projection gradient 0 = not computed (p.grad_projections null), 1 = four
// float reductions per voxel-view into grad_projections.
//
// A warp owns one (x, y) column and 32*KZ of its voxels along z.  Views go in
// passes of 32: lane j evaluates the column geometry of view a0+j (and, at
// the end of the pass, its chain rule).  The warp walks the pass's views
// kBpGroup at a time with that view's geometry broadcast by shuffles; per
// view every lane first issues the loads of its KZ taps together (an
// out-of-range tap loads the row's first quad and is masked), then adds its
// voxels' four products into registers.  The group's 4 x kBpGroup sums are
// reduced over the warp at once (warp_transpose_sum) and kept by the lane
// that owns the view; after the pass all 32 lanes apply the chain rule at
// once.
template <int KZ, int GP>
__global__ void __launch_bounds__(256) bp_backward_kernel(BpArgs p) {
    constexpr int G = kBpGroup;
    __shared__ double s_terms[8][32][8];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cols_x = (p.W + 7) >> 3;
    const long long block_id = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    const BpTile tile = bp_tile(block_id, cols_x, p.H, bp_super(8), bp_super(1));
    const int y = tile.ty;
    const int x = tile.tx * 8 + warp;
    const int zbase = tile.zb * 32 * KZ;
    const long long nblocks = (long long)gridDim.x * gridDim.y;
    const bool col_ok = x < p.W;
    const float vx = (x - p.W * 0.5f) * p.voxel_size + p.off_x;
    const float vy = (y - p.H * 0.5f) * p.voxel_size + p.off_y;
    const float ip = p.inv_pixel;

    float gval[KZ], pz[KZ];
#pragma unroll
    for (int k = 0; k < KZ; ++k) {
        const int z = zbase + lane + 32 * k;
        pz[k] = (z - p.D * 0.5f) * p.voxel_size + p.off_z;
        gval[k] = (col_ok && z < p.D) ? p.grad_volume[((long long)z * p.H + y) * p.W + x] : 0.0f;
    }
    const int zlimit = p.D - zbase - lane;
    const uint32_t vcount = (uint32_t)max(p.V - 1, 0);
    f32x2 pz2[KZ / 2 > 0 ? KZ / 2 : 1];
#pragma unroll
    for (int k = 0; k + 1 < KZ; k += 2) pz2[k / 2] = pack2(pz[k], pz[k + 1]);
    const f32x2 ip2 = pack2(p.inv_pixel, p.inv_pixel);
    const f32x2 magic2 = pack2(kFloorMagic, kFloorMagic);

    for (int a0 = 0; a0 < p.A; a0 += 32) {
        const int nv = min(32, p.A - a0);
        // the values the z loop needs from lane j's view (the rest of its
        // geometry is recomputed by the same lane for the chain rule)
        float my_t = 0.f, my_dsv = 0.f, my_v0 = 0.f, my_fu = 0.f, my_w = 0.f;
        int my_ui = 0;
        bool my_ok = false;
        if (lane < nv) {
            const ColumnGrad g = column_grad(p.vt[a0 + lane], vx, vy, col_ok, p);
            my_ok = g.ok;
            my_t = g.t;
            my_dsv = g.ds_v;
            my_v0 = g.v0;
            my_fu = g.fu;
            my_w = g.w;
            my_ui = g.ui;
        }
        const unsigned valid_mask = __ballot_sync(FULL, my_ok);
        // this lane's view: its four z-sums over the warp's voxels
        float m_iu = 0.f, m_iv = 0.f, m_ivdv = 0.f, m_int = 0.f;
        for (int b = 0; b < nv; b += G) {
            float acc[4 * G];
#pragma unroll
            for (int i = 0; i < 4 * G; ++i) acc[i] = 0.0f;
#pragma unroll
            for (int i = 0; i < G; ++i) {
                const int j = b + i;
                if (!((valid_mask >> j) & 1u)) continue;  // warp-uniform
                const float t = __shfl_sync(FULL, my_t, j);
                const float dsv = __shfl_sync(FULL, my_dsv, j);
                const float v0 = __shfl_sync(FULL, my_v0, j);
                const float fu = __shfl_sync(FULL, my_fu, j);
                const int ui = __shfl_sync(FULL, my_ui, j);
                const int a = a0 + j;
                const ulonglong2* __restrict__ rq =
                    reinterpret_cast<const ulonglong2*>(p.pquads) + (a * (p.U - 1) + ui) * (p.V - 1);
                float w = 0.0f;
                float* __restrict__ gp = nullptr;
                if (GP) {
                    w = __shfl_sync(FULL, my_w, j);
                    gp = p.grad_projections + ((long long)a * p.U + ui) * p.V;
                }
                ulonglong2 q[KZ];
                float fvk[KZ], dvk[KZ];
                int vik[KZ];
                bool okk[KZ];
                // z voxels in pairs: v_idx and its floor split as packed f32x2;
                // a tap is valid iff its floor, as an unsigned index, is below V-1
                auto setup = [&](int k, float dv, uint32_t biased, float fv) {
                    const uint32_t vi = biased - kFloorMagicBits;
                    okk[k] = 32 * k < zlimit && vi < vcount;
                    vik[k] = okk[k] ? (int)vi : 0;
                    fvk[k] = fv;
                    dvk[k] = dv;
                    q[k] = __ldg(rq + vik[k]);
                };
                if constexpr (KZ % 2 == 0) {
                    const f32x2 t2 = pack2(t, t), d2 = pack2(dsv, dsv), o2 = pack2(v0, v0);
#pragma unroll
                    for (int k = 0; k < KZ; k += 2) {
                        const f32x2 dv2 = sub2(pz2[k / 2], d2);
                        const f32x2 vx2 = fma2(fma2(t2, dv2, d2), ip2, o2);
                        const f32x2 f2 = add2_rd(vx2, magic2);
                        const float2 fr = unpack2(sub2(vx2, sub2(f2, magic2)));
                        const uint2 bits = unpack2_bits(f2);
                        const float2 dv = unpack2(dv2);
                        setup(k, dv.x, bits.x, fr.x);
                        setup(k + 1, dv.y, bits.y, fr.y);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < KZ; ++k) {
                        const float dv = pz[k] - dsv;
                        const float v_phys = dsv + t * dv;
                        const FloorSplit fs = floor_split(v_phys * ip + v0);
                        setup(k, dv, fs.biased, fs.frac);
                    }
                }
#pragma unroll
                for (int k = 0; k < KZ; ++k) {
                    if (okk[k]) {
                        const float fv = fvk[k], dv = dvk[k];
                        const int vi = vik[k];
                        // column pairs (rows u, u+1) at v and v+1: the lerp along v
                        // and the difference along v as packed pairs
                        const float2 e = unpack2(lerp2(q[k].x, q[k].y, pack2(fv, fv)));
                        const float2 d = unpack2(sub2(q[k].y, q[k].x));
                        const float2 c0 = unpack2(q[k].x), c1 = unpack2(q[k].y);
                        const float interp = lerpf(e.x, e.y, fu);
                        const float iu = lerpf(c0.y - c0.x, c1.y - c1.x, fv);
                        const float iv = lerpf(d.x, d.y, fu);
                        const float g = gval[k];
                        acc[4 * i + 0] = fmaf(g, iu, acc[4 * i + 0]);
                        acc[4 * i + 1] = fmaf(g, iv, acc[4 * i + 1]);
                        acc[4 * i + 2] = fmaf(g * iv, dv, acc[4 * i + 2]);
                        acc[4 * i + 3] = fmaf(g, interp, acc[4 * i + 3]);
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
            }
            // lane 4i+q: sum q of view b+i; the view's owner (lane b+i) keeps its four
            const float total = warp_transpose_sum<4 * G>(acc, lane);
            const int src = 4 * ((lane - b) & (G - 1));
            const float s_iu = __shfl_sync(FULL, total, src + 0);
            const float s_iv = __shfl_sync(FULL, total, src + 1);
            const float s_ivdv = __shfl_sync(FULL, total, src + 2);
            const float s_int = __shfl_sync(FULL, total, src + 3);
            if (lane >= b && lane < b + G) {
                m_iu = s_iu;
                m_iv = s_iv;
                m_ivdv = s_ivdv;
                m_int = s_int;
            }
        }
        float terms[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (my_ok) {
            const ColumnGrad g = column_grad(p.vt[a0 + lane], vx, vy, col_ok, p);
            column_terms(g, m_iu, m_iv, m_ivdv, m_int, ip, terms);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) s_terms[warp][lane][k] = (double)terms[k];
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
// 0.46 / 0.36 / 0.52 / 0.52 ms, 17.0 / 13.7 / 14.5 / 15.5 ms (before the
// super-tile order).  Backward at 256^3 / 360 x 384^2 (current kernel),
// KZ = 2 / 4 / 8: 12.6 / 10.5 / 10.9 ms without the projection gradient,
// 22.9 / 25.1 / 28.7 ms with it.
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
    DGC_TRACE(p.grad_projections ? "bp_backward_kernel<gp>" : "bp_backward_kernel", s);
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
