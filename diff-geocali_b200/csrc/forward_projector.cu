// forward_projector.cu -- ray-driven cone-beam forward projector and its
// hand-written backward, for sm_100a.
//
// Semantics follow the reference kernels of TomSHINING/diff-geoCali,
// csrc/src_cbct_forwardprojector_cuda.cu:
//   ray set-up        make_source_only_ray 115-170, intersect_aabb 86-112
//   fixed-step march  258-339 (t from t_min by repeated FP32 adds of step while
//                     t <= t_max, trilinear samples with clamped neighbours)
//   backward          342-528 (adjoint scatter, spatial-gradient sums, entry-
//                     slab chain rule, normalisation chain, per-view terms)
//
// B200 design (not the reference's):
//   * Z-fastest quad layout.  Per call the volume is re-laid out into an
//     edge-replicated copy Q[y+1][x+1][z+1] = float4(v(z,y,x), v(z,y+1,x),
//     v(z,y,x+1), v(z,y+1,x+1)) with z the fastest index.  The detector's V
//     axis is parallel to z for every view, so the 32 lanes of a warp -- 32
//     consecutive detector rows of one column -- sample nearly the same (x, y)
//     at consecutive z: each 16-byte load of a warp touches a few contiguous
//     lines at every view angle, and the z+1 quad is the next element.
//   * Edge replication replaces the reference's per-corner clamping: with the
//     one-voxel pad, any coordinate in [-1, n) addresses valid quads whose
//     out-of-range neighbours equal the edge value, which is exactly what the
//     clamped reference reads.  A ray whose sample segment stays inside that
//     range (checked once per ray) runs a loop without clamps; others clamp.
//   * floor() runs on the FP32 add pipe (round-down add of 1.5*2^23).
//   * CTAs are ordered u-tile fastest, then view, then detector-row band.  The
//     rays of one band are nearly horizontal and cross only a z-slab of the
//     volume, so the many views in flight share a slab that stays in L2.
//   * Geometry gradients are reduced per CTA in FP64 with warp shuffles and a
//     fixed-order tree, then per view over CTAs in a second fixed-order pass:
//     the eight per-view gradients are bitwise reproducible.
//   * The volume gradient is scattered into an edge-padded z-fastest buffer
//     (consecutive lanes hit consecutive addresses) and folded back onto the
//     clamped edge voxels afterwards (the sums of the reference's clamped-index
//     atomics).
#include <cstdlib>
#include <mutex>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "forward_projector.cuh"
#include "tma.cuh"

namespace dgc {

// ---------------------------------------------------------------------------
// Volume re-layout: [D][H][W] -> Z-fastest edge-replicated quads
// ---------------------------------------------------------------------------

// One 32 x 32 (x, z) tile of the quads at padded row yp: block (32, 8).
__device__ __forceinline__ void quads_tile(const float* __restrict__ vol, int D, int H, int W,
                                           float4* __restrict__ Q, int bx, int by,
                                           float4 (&tile)[32][33]) {
    const int xtiles = (W + 1 + 31) / 32;
    const int yp = bx / xtiles;
    const int xp0 = (bx - yp * xtiles) * 32;
    const int zp0 = by * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    {
        const int xp = xp0 + tx;
        const int x0 = min(max(xp - 1, 0), W - 1), x1 = min(xp, W - 1);
        const int y0 = min(max(yp - 1, 0), H - 1), y1 = min(yp, H - 1);
        for (int zl = ty; zl < 32; zl += 8) {
            const int z = min(max(zp0 + zl - 1, 0), D - 1);
            const float* plane = vol + (long long)z * H * W;
            // (x0,y0), (x0,y1), (x1,y0), (x1,y1): the y-pairs of each x are
            // 64-bit halves, the operands of the packed lerps
            tile[zl][tx] = make_float4(__ldg(plane + (long long)y0 * W + x0),
                                       __ldg(plane + (long long)y1 * W + x0),
                                       __ldg(plane + (long long)y0 * W + x1),
                                       __ldg(plane + (long long)y1 * W + x1));
        }
    }
    __syncthreads();
    const int zp = zp0 + tx;
    for (int xl = ty; xl < 32; xl += 8) {
        const int xp = xp0 + xl;
        if (xp <= W && zp <= D + 1)
            Q[((long long)yp * (W + 1) + xp) * (D + 2) + zp] = tile[tx][xl];
    }
}

// grid: x = ceil((W+1)/32) * (H+1), y = ceil((D+2)/32); block (32, 8)
__global__ void build_volume_quads_kernel(const float* __restrict__ vol, int D, int H, int W,
                                          float4* __restrict__ Q) {
    __shared__ float4 tile[32][33];
    quads_tile(vol, D, H, W, Q, blockIdx.x, blockIdx.y, tile);
}

int build_volume_quads(const float* vol, int D, int H, int W, float4* quads, cudaStream_t s) {
    DGC_TRACE("build_volume_quads", s);
    const dim3 grid((unsigned)(ceil_div(W + 1, 32) * (long long)(H + 1)), (unsigned)ceil_div(D + 2, 32));
    build_volume_quads_kernel<<<grid, dim3(32, 8), 0, s>>>(vol, D, H, W, quads);
    DGC_LAUNCH_CHECK("build_volume_quads");
    return DGC_OK;
}

// Z-pair layout of the forward's pair arm: P[(yq*(W+2) + xq)*(D+1) + zp] =
// (v(z0, y, x), v(z1, y, x)) with y = yq-1, x = xq-1, z0 = zp-1, z1 = zp, all
// clamped to the volume -- half the quads' bytes (8 per padded voxel).  A
// cell's eight corners are four pairs (x and y neighbours at +(D+1) and
// +(W+2)(D+1)), regrouped in registers into the two quads of the cell, so
// the interpolation is bitwise the quad arm's.
// grid: x = ceil((W+2)/32) * (H+2), y = ceil((D+1)/32); block (32, 8)
__global__ void build_volume_pairs_kernel(const float* __restrict__ vol, int D, int H, int W,
                                          float2* __restrict__ P) {
    __shared__ float2 tile[32][33];
    const int xtiles = (W + 2 + 31) / 32;
    const int yq = blockIdx.x / xtiles;
    const int xq0 = (blockIdx.x - yq * xtiles) * 32;
    const int zp0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    {
        const int x = min(max(xq0 + tx - 1, 0), W - 1);
        const int y = min(max(yq - 1, 0), H - 1);
        for (int zl = ty; zl < 32; zl += 8) {
            const int z0 = min(max(zp0 + zl - 1, 0), D - 1), z1 = min(zp0 + zl, D - 1);
            tile[zl][tx] = make_float2(__ldg(vol + ((long long)z0 * H + y) * W + x),
                                       __ldg(vol + ((long long)z1 * H + y) * W + x));
        }
    }
    __syncthreads();
    const int zp = zp0 + tx;
    for (int xl = ty; xl < 32; xl += 8) {
        const int xq = xq0 + xl;
        if (xq <= W + 1 && zp <= D)
            P[((long long)yq * (W + 2) + xq) * (D + 1) + zp] = tile[tx][xl];
    }
}

int build_volume_pairs(const float* vol, int D, int H, int W, float2* pairs, cudaStream_t s) {
    DGC_TRACE("build_volume_pairs", s);
    const dim3 grid((unsigned)(ceil_div(W + 2, 32) * (long long)(H + 2)), (unsigned)ceil_div(D + 1, 32));
    build_volume_pairs_kernel<<<grid, dim3(32, 8), 0, s>>>(vol, D, H, W, pairs);
    DGC_LAUNCH_CHECK("build_volume_pairs");
    return DGC_OK;
}

// ---------------------------------------------------------------------------
// Per-view and per-ray set-up (reference arithmetic, kept expression for
// expression so that t_min / t_max -- and with them the FP32 sample count --
// agree with the reference kernel).  Every multiply-add is written out as
// fmaf / __fmul_rn: left to the compiler, a*b - c*d may be contracted
// differently in different kernels (depending on which products a kernel
// reuses), and the forward, backward, fused and batched kernels must march
// bitwise the same rays.
// ---------------------------------------------------------------------------

struct ViewGeo {
    float c, s, sod, dn, u0, v0, ox, oy, oz;
};

__device__ __forceinline__ void load_view(const Geometry& g, int a, ViewGeo& vg) {
    const float beta = g.angles[a];
    vg.c = cosf(beta);
    vg.s = sinf(beta);
    vg.sod = g.sod[a];
    vg.dn = vg.sod - g.sid[a];
    vg.u0 = g.det_u0[a];
    vg.v0 = g.det_v0[a];
    vg.ox = fmaf(-vg.sod, vg.s, g.src_x[a]);
    vg.oy = fmaf(vg.sod, vg.c, g.src_y[a]);
    vg.oz = g.src_z[a];
}

struct RaySetup {
    float dx, dy, dz;
    float len;
    float tmin, tmax;
    int entry_axis;
    bool ok;   // ray length > 1e-8
    bool hit;  // intersects the volume box
};

__device__ __forceinline__ bool slab(float origin, float direction, float lo, float hi, int axis,
                                     float& tmin, float& tmax, int& entry) {
    if (fabsf(direction) < 1e-12f) return origin >= lo && origin <= hi;
    const float inv = 1.0f / direction;
    float t1 = (lo - origin) * inv;
    float t2 = (hi - origin) * inv;
    if (t1 > t2) {
        const float tmp = t1;
        t1 = t2;
        t2 = tmp;
    }
    if (t1 > tmin) {
        tmin = t1;
        entry = axis;
    }
    tmax = fminf(tmax, t2);
    return tmax >= tmin;
}

__device__ __forceinline__ RaySetup setup_ray(const ViewGeo& vg, int u, int v, const FpArgs& p) {
    RaySetup r;
    const float u_phys = (u - vg.u0) * p.pixel_size;
    const float v_phys = (v - vg.v0) * p.pixel_size;
    const float tx = fmaf(u_phys, vg.c, -__fmul_rn(vg.dn, vg.s));
    const float ty = fmaf(u_phys, vg.s, __fmul_rn(vg.dn, vg.c));
    const float tz = v_phys;
    const float rx = tx - vg.ox, ry = ty - vg.oy, rz = tz - vg.oz;
    r.len = sqrtf(fmaf(rz, rz, fmaf(rx, rx, __fmul_rn(ry, ry))));
    r.ok = r.len > 1e-8f;
    r.hit = false;
    r.dx = r.dy = r.dz = 0.0f;
    r.tmin = 0.0f;
    r.tmax = 0.0f;
    r.entry_axis = -1;
    if (!r.ok) return r;
    const float inv_len = 1.0f / r.len;
    r.dx = rx * inv_len;
    r.dy = ry * inv_len;
    r.dz = rz * inv_len;
    // (-n/2 - 1/2) and (n/2 - 1/2) are exact in FP32 for every n < 2^23
    const float bxl = fmaf(-p.W * 0.5f - 0.5f, p.voxel_size, p.off_x);
    const float byl = fmaf(-p.H * 0.5f - 0.5f, p.voxel_size, p.off_y);
    const float bzl = fmaf(-p.D * 0.5f - 0.5f, p.voxel_size, p.off_z);
    const float bxh = fmaf(p.W * 0.5f - 0.5f, p.voxel_size, p.off_x);
    const float byh = fmaf(p.H * 0.5f - 0.5f, p.voxel_size, p.off_y);
    const float bzh = fmaf(p.D * 0.5f - 0.5f, p.voxel_size, p.off_z);
    float tmin = 0.0f, tmax = FLT_MAX;
    int entry = -1;
    r.hit = slab(vg.ox, r.dx, bxl, bxh, 0, tmin, tmax, entry) &&
            slab(vg.oy, r.dy, byl, byh, 1, tmin, tmax, entry) &&
            slab(vg.oz, r.dz, bzl, bzh, 2, tmin, tmax, entry) && tmax >= tmin;
    r.tmin = tmin;
    r.tmax = tmax;
    r.entry_axis = entry;
    return r;
}

// Bound on the number of FP32 recurrence steps: the reference's loop would
// not terminate if t + step == t; the bound is far above the count of every
// advancing recurrence.
__device__ __forceinline__ int step_bound(const RaySetup& r, float step) {
    const float n = (r.tmax - r.tmin) / step;
    return n < 1.0e9f ? 2 * (int)n + 16 : 2000000000;
}

// True when every t of the ray's recurrence satisfies |t| < 2^22 * step: then
// ulp(t) < step, each t += step advances t by more than step/2 and the loop
// ends by itself, so it may run without the iteration counter.
__device__ __forceinline__ bool steps_advance(const RaySetup& r, float step) {
    const float lim = 4194304.0f * step;
    return fabsf(r.tmin) < lim && fabsf(r.tmax) + step < lim;
}

// Voxel coordinate of a world position along one axis.
//   forward (fp.cu:326-328): (p - off) / voxel + n/2
//   backward (fp.cu:425-427): (p - off) * (1/voxel) + n/2
// For a power-of-two voxel size both are one fused multiply-add.
// OFF = false skips the subtraction of a zero ROI offset (exact: p - 0 = p).
template <bool DIV, bool OFF = true>
__device__ __forceinline__ float to_voxel(float pos, float off, float voxel, float inv_voxel,
                                          float half) {
    const float q = OFF ? pos - off : pos;
    if (DIV) return __fdiv_rn(q, voxel) + half;
    return fmaf(q, inv_voxel, half);
}

// True when every sample coordinate of the ray lies in [-1, n) with a 0.05
// margin, i.e. the loop may address the padded layouts without clamping.
// Samples lie between the box entry and exit points, so the two end points
// bound them (up to FP32 rounding, far below the margin).
template <bool DIV>
__device__ __forceinline__ bool ray_inside_pad(const RaySetup& r, const ViewGeo& vg,
                                               const FpArgs& p) {
    const float hx = p.W * 0.5f, hy = p.H * 0.5f, hz = p.D * 0.5f;
    const float x0 = to_voxel<DIV>(fmaf(r.tmin, r.dx, vg.ox), p.off_x, p.voxel_size, p.inv_voxel, hx);
    const float x1 = to_voxel<DIV>(fmaf(r.tmax, r.dx, vg.ox), p.off_x, p.voxel_size, p.inv_voxel, hx);
    const float y0 = to_voxel<DIV>(fmaf(r.tmin, r.dy, vg.oy), p.off_y, p.voxel_size, p.inv_voxel, hy);
    const float y1 = to_voxel<DIV>(fmaf(r.tmax, r.dy, vg.oy), p.off_y, p.voxel_size, p.inv_voxel, hy);
    const float z0 = to_voxel<DIV>(fmaf(r.tmin, r.dz, vg.oz), p.off_z, p.voxel_size, p.inv_voxel, hz);
    const float z1 = to_voxel<DIV>(fmaf(r.tmax, r.dz, vg.oz), p.off_z, p.voxel_size, p.inv_voxel, hz);
    const float lo = -0.95f;
    return fminf(x0, x1) >= lo && fmaxf(x0, x1) <= p.W - 0.05f && fminf(y0, y1) >= lo &&
           fmaxf(y0, y1) <= p.H - 0.05f && fminf(z0, z1) >= lo && fmaxf(z0, z1) <= p.D - 0.05f;
}

struct Cell {
    uint32_t bx, by, bz;  // biased floors (kFloorMagicBits + floor)
    float fx, fy, fz;
};

// Cell of a sample.  CLAMP limits the coordinate to [-1, n-1]: beyond it both
// neighbours are edge replicas, so the interpolated value is unchanged.
template <bool CLAMP>
__device__ __forceinline__ Cell locate(float x, float y, float z, const FpArgs& p) {
    if (CLAMP) {
        x = fminf(fmaxf(x, -1.0f), (float)(p.W - 1));
        y = fminf(fmaxf(y, -1.0f), (float)(p.H - 1));
        z = fminf(fmaxf(z, -1.0f), (float)(p.D - 1));
    }
    const FloorSplit sx = floor_split(x), sy = floor_split(y), sz = floor_split(z);
    Cell c;
    c.bx = sx.biased;
    c.by = sy.biased;
    c.bz = sz.biased;
    c.fx = sx.frac;
    c.fy = sy.frac;
    c.fz = sz.frac;
    return c;
}

// Loop invariants of the packed (x, y) sample position.
struct XYPacks {
    f32x2 dxy, oxy, offxy, inv2, hxy, magic2;
};

__device__ __forceinline__ XYPacks make_xy_packs(const RaySetup& r, const ViewGeo& vg,
                                                 const FpArgs& p) {
    XYPacks k;
    k.dxy = pack2(r.dx, r.dy);
    k.oxy = pack2(vg.ox, vg.oy);
    k.offxy = pack2(p.off_x, p.off_y);
    k.inv2 = pack2(p.inv_voxel, p.inv_voxel);
    k.hxy = pack2(p.W * 0.5f, p.H * 0.5f);
    k.magic2 = pack2(kFloorMagic, kFloorMagic);
    return k;
}

// Cell of the sample at t.  With PACK, no clamping and the multiplying voxel
// conversion, x and y run as packed pairs (fma.rn / sub.rn / add.rm on
// f32x2): lane by lane the same IEEE operations as the scalar path, so the
// cell and weights are bitwise those of locate(to_voxel(...)).  Measured on
// the forward sum 1-3 % faster; in the gradient marches (more live values)
// the scalar form is faster, so they keep it.
template <bool CLAMP, bool DIV, bool OFF, bool PACK>
__device__ __forceinline__ Cell sample_cell(float t, const RaySetup& r, const ViewGeo& vg,
                                            const FpArgs& p, const XYPacks& k) {
    const float hz = p.D * 0.5f;
    if constexpr (PACK && !CLAMP && !DIV) {
        const f32x2 pxy = fma2(pack2(t, t), k.dxy, k.oxy);
        const f32x2 vxy = fma2(OFF ? sub2(pxy, k.offxy) : pxy, k.inv2, k.hxy);
        const f32x2 fxy = add2_rd(vxy, k.magic2);
        const float2 frac = unpack2(sub2(vxy, sub2(fxy, k.magic2)));
        const uint2 bits = unpack2_bits(fxy);
        const FloorSplit sz =
            floor_split(to_voxel<false, OFF>(fmaf(t, r.dz, vg.oz), p.off_z, p.voxel_size,
                                             p.inv_voxel, hz));
        Cell c;
        c.bx = bits.x;
        c.by = bits.y;
        c.bz = sz.biased;
        c.fx = frac.x;
        c.fy = frac.y;
        c.fz = sz.frac;
        return c;
    } else {
        const float hx = p.W * 0.5f, hy = p.H * 0.5f;
        return locate<CLAMP>(
            to_voxel<DIV, OFF>(fmaf(t, r.dx, vg.ox), p.off_x, p.voxel_size, p.inv_voxel, hx),
            to_voxel<DIV, OFF>(fmaf(t, r.dy, vg.oy), p.off_y, p.voxel_size, p.inv_voxel, hy),
            to_voxel<DIV, OFF>(fmaf(t, r.dz, vg.oz), p.off_z, p.voxel_size, p.inv_voxel, hz), p);
    }
}

__device__ __forceinline__ uint32_t quad_index(const Cell& c, const FpArgs& p) {
    return c.bz + c.bx * p.zq_x + c.by * p.zq_y + p.zq_bias;
}

// The two quads (z and z+1) of cell qi.  Consecutive samples of a ray often
// stay in one cell (about half of them at step 0.5 voxel along an axis), and
// then read the same 32 bytes: those keep the previous sample's registers and
// issue no load.  Bitwise the same values as loading every sample.  Used by
// the value march only: it takes the forward at 256^3 / 360 x 384^2 from
// 40.1 to 38.7 ms and the batched forward of that instance plus its half
// from 50.9 to 48.1 ms, while the gradient marches, which hold more live
// values, slowed by 2-17 % with it.
struct CellQuads {
    uint32_t qi = 0xffffffffu;  // no quad index reaches 2^32 - 1
    ulonglong2 q0 = {0ull, 0ull}, q1 = {0ull, 0ull};
};

__device__ __forceinline__ void load_cell(const ulonglong2* __restrict__ Q, uint32_t qi,
                                          CellQuads& cq) {
    if (qi != cq.qi) {
        cq.q0 = __ldg(Q + qi);
        cq.q1 = __ldg(Q + qi + 1);
        cq.qi = qi;
    }
}

// Sum of the trilinear samples along the ray (fp.cu:321-335).  The quads
// hold the y-pairs of x0 and x1 as 64-bit halves, so the interpolation runs
// as packed pairs: along x for (y0, y1) at z0 and z1, along z, then along y.
// UNROLL: the march loop unrolled by the compiler (1 or 2; the same samples
// and sums either way, a tuned dimension of the forward).
template <bool CLAMP, bool DIV, bool OFF, bool GUARD = true, int UNROLL = 1>
__device__ __forceinline__ float march_sum(const RaySetup& r, const ViewGeo& vg, const FpArgs& p) {
    const ulonglong2* __restrict__ Q = reinterpret_cast<const ulonglong2*>(p.quads);
    const XYPacks k = make_xy_packs(r, vg, p);
    const int nmax = step_bound(r, p.step_size);
    float acc = 0.0f;
    float t = r.tmin;
    int n = 0;
    CellQuads cq;
#pragma unroll UNROLL
    for (; t <= r.tmax && (!GUARD || n < nmax); t += p.step_size, n += GUARD ? 1 : 0) {
        const Cell c = sample_cell<CLAMP, DIV, OFF, true>(t, r, vg, p, k);
        load_cell(Q, quad_index(c, p), cq);
        const ulonglong2 q0 = cq.q0, q1 = cq.q1;
        const f32x2 wx = pack2(c.fx, c.fx);
        const f32x2 e0 = lerp2(q0.x, q0.y, wx);  // (y0, y1) at z0
        const f32x2 e1 = lerp2(q1.x, q1.y, wx);  // (y0, y1) at z1
        const float2 e = unpack2(lerp2(e0, e1, pack2(c.fz, c.fz)));
        acc += lerpf(e.x, e.y, c.fy);
    }
    return acc;
}

// CTA -> (u tile, view, v band): u tile fastest, then view, then band.
struct TileCoord {
    int a, tu, tv;
};

__host__ __device__ __forceinline__ long long fp_tiles_per_view_dev(int U, int V, int tu) {
    return (long long)((U + tu - 1) / tu) * ((V + 256 / tu - 1) / (256 / tu));
}

// With p.view_block = B > 0, inside a band the views go in blocks of B and,
// inside a block, the view runs fastest, then the u tile: the CTAs in flight
// then cover B views of a few u tiles instead of every u tile of a few views
// (a smaller set of volume cells, shared across views; a tuned dimension of
// the forward).  The order changes no result.
__device__ __forceinline__ TileCoord tile_coord(const FpArgs& p, int tiles_u) {
    int b = blockIdx.x;
    TileCoord tc;
    if (p.view_block <= 0) {
        tc.tu = b % tiles_u;
        b /= tiles_u;
        tc.a = b % p.A;
        tc.tv = b / p.A;
        return tc;
    }
    const int per_band = tiles_u * p.A;
    tc.tv = b / per_band;
    int r = b - tc.tv * per_band;
    const int block_tiles = p.view_block * tiles_u;
    const int vb = r / block_tiles;
    r -= vb * block_tiles;
    const int nv = min(p.view_block, p.A - vb * p.view_block);
    tc.a = vb * p.view_block + r % nv;
    tc.tu = r / nv;
    return tc;
}

// ---------------------------------------------------------------------------
// Forward kernel
// ---------------------------------------------------------------------------

// Ray of this thread in a TU x (256/TU) tile.  WU = 1: warps run along V (32
// consecutive rows of one column).  WU > 1: a warp takes a patch of WU
// columns x 32/WU rows (lanes along V first).
template <int TU, int WU = 1>
__device__ __forceinline__ void tile_ray(const TileCoord& tc, int& u, int& v) {
    constexpr int TV = 256 / TU;
    constexpr int WARPS_V = TV / 32;
    static_assert(TV % 32 == 0, "rows per CTA must be whole warps");
    static_assert(TU % WU == 0 && 32 % WU == 0, "warp patches must tile the CTA");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if constexpr (WU == 1) {
        u = tc.tu * TU + warp / WARPS_V;
        v = tc.tv * TV + (warp % WARPS_V) * 32 + lane;
    } else {
        constexpr int ROWS = 32 / WU;
        u = tc.tu * TU + (warp % (TU / WU)) * WU + lane / ROWS;
        v = tc.tv * TV + (warp / (TU / WU)) * ROWS + lane % ROWS;
    }
}

// Line integral of one ray, written to p.projections.
template <bool DIV, bool OFF, int UNROLL = 1>
__device__ __forceinline__ void forward_ray(const FpArgs& p, const ViewGeo& vg, int a, int u,
                                            int v) {
    const RaySetup r = setup_ray(vg, u, v, p);
    float integral = 0.0f;
    if (r.ok && r.hit) {
        const bool inside = ray_inside_pad<DIV>(r, vg, p);
        if (steps_advance(r, p.step_size))
            integral = inside ? march_sum<false, DIV, OFF, false, UNROLL>(r, vg, p)
                              : march_sum<true, DIV, OFF, false, UNROLL>(r, vg, p);
        else
            integral = inside ? march_sum<false, DIV, OFF, true, UNROLL>(r, vg, p)
                              : march_sum<true, DIV, OFF, true, UNROLL>(r, vg, p);
        integral *= p.step_size;
    }
    p.projections[((long long)a * p.U + u) * p.V + v] = integral;
}

// A CTA owns TU detector columns x (256/TU) rows of one view.
template <int TU, bool DIV, bool OFF, int UNROLL = 1>
__global__ void __launch_bounds__(256) fp_forward_kernel(FpArgs p) {
    __shared__ ViewGeo s_view;
    const int tiles_u = (p.U + TU - 1) / TU;
    const TileCoord tc = tile_coord(p, tiles_u);
    if (threadIdx.x == 0) load_view(p.g, tc.a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    int u, v;
    // with view blocks (the order for volumes beyond L2) warps take 4 x 8 ray
    // patches: 671.3 -> 658.9 ms at 512^3 / 720 x 768^2, while at 256^3 /
    // 720 x 384^2 the 4 x 8 patches are 1.3 % slower than 1 x 32 columns (the
    // autotuner's view-block arms carry the patches, so its timings include
    // them; the projections are the same)
    if (TU % 4 == 0 && p.view_block > 0) tile_ray<TU, (TU % 4 == 0 ? 4 : 1)>(tc, u, v);
    else tile_ray<TU>(tc, u, v);
    if (u >= p.U || v >= p.V) return;
    forward_ray<DIV, OFF, UNROLL>(p, vg, tc.a, u, v);
}

// ---------------------------------------------------------------------------
// Forward kernel, pair arm: the volume as z-pairs (half the quads' footprint)
// ---------------------------------------------------------------------------

// march_sum over the z-pair layout: the same samples, cells and packed lerps
// (the four pairs of a cell regrouped into its two quads), four 8-byte loads
// per new cell instead of two 16-byte ones.
template <bool CLAMP, bool DIV, bool OFF, bool GUARD = true>
__device__ __forceinline__ float march_sum_pairs(const RaySetup& r, const ViewGeo& vg,
                                                 const FpArgs& p) {
    const unsigned long long* __restrict__ P =
        reinterpret_cast<const unsigned long long*>(p.quads);
    const XYPacks k = make_xy_packs(r, vg, p);
    const int nmax = step_bound(r, p.step_size);
    const uint32_t sx = (uint32_t)(p.D + 1), sy = (uint32_t)(p.W + 2) * (uint32_t)(p.D + 1);
    const uint32_t bias = (1u + sx + sy) - kFloorMagicBits * (1u + sx + sy);
    float acc = 0.0f;
    float t = r.tmin;
    int n = 0;
    CellQuads cq;
#pragma unroll 1
    for (; t <= r.tmax && (!GUARD || n < nmax); t += p.step_size, n += GUARD ? 1 : 0) {
        const Cell c = sample_cell<CLAMP, DIV, OFF, true>(t, r, vg, p, k);
        const uint32_t pi = c.bz + c.bx * sx + c.by * sy + bias;
        if (pi != cq.qi) {
            const float2 p00 = unpack2(__ldg(P + pi)), p10 = unpack2(__ldg(P + pi + sx));
            const float2 p01 = unpack2(__ldg(P + pi + sy)), p11 = unpack2(__ldg(P + pi + sy + sx));
            cq.q0 = make_ulonglong2(pack2(p00.x, p01.x), pack2(p10.x, p11.x));
            cq.q1 = make_ulonglong2(pack2(p00.y, p01.y), pack2(p10.y, p11.y));
            cq.qi = pi;
        }
        const ulonglong2 q0 = cq.q0, q1 = cq.q1;
        const f32x2 wx = pack2(c.fx, c.fx);
        const f32x2 e0 = lerp2(q0.x, q0.y, wx);
        const f32x2 e1 = lerp2(q1.x, q1.y, wx);
        const float2 e = unpack2(lerp2(e0, e1, pack2(c.fz, c.fz)));
        acc += lerpf(e.x, e.y, c.fy);
    }
    return acc;
}

template <int TU, bool DIV, bool OFF>
__global__ void __launch_bounds__(256) fp_forward_pairs_kernel(FpArgs p) {
    __shared__ ViewGeo s_view;
    const int tiles_u = (p.U + TU - 1) / TU;
    const TileCoord tc = tile_coord(p, tiles_u);
    if (threadIdx.x == 0) load_view(p.g, tc.a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    int u, v;
    tile_ray<TU>(tc, u, v);
    if (u >= p.U || v >= p.V) return;
    const RaySetup r = setup_ray(vg, u, v, p);
    float integral = 0.0f;
    if (r.ok && r.hit) {
        const bool inside = ray_inside_pad<DIV>(r, vg, p);
        if (steps_advance(r, p.step_size))
            integral = inside ? march_sum_pairs<false, DIV, OFF, false>(r, vg, p)
                              : march_sum_pairs<true, DIV, OFF, false>(r, vg, p);
        else
            integral = inside ? march_sum_pairs<false, DIV, OFF>(r, vg, p)
                              : march_sum_pairs<true, DIV, OFF>(r, vg, p);
        integral *= p.step_size;
    }
    p.projections[((long long)tc.a * p.U + u) * p.V + v] = integral;
}

// ---------------------------------------------------------------------------
// Forward kernel, TMA arm: volume bricks staged in shared memory
// ---------------------------------------------------------------------------
//
// The CTA's 256 rays (one view, 8 detector columns x 32 rows) form a thin
// bundle that runs along one horizontal axis m (x or y, whichever the bundle's
// central ray follows more).  Its march is cut into slabs of L cells along m;
// for each slab one thread issues a 3-D cp.async.bulk.tensor copy of the
// quads under the bundle -- L cells along m, kTmaO across, kTmaZ along z, a
// box bounded from the bundle's four corner rays at the slab's two faces --
// into one of two shared-memory stages, so the copy of slab i+1 overlaps the
// samples of slab i.  Every thread marches its own ray (the same FP32
// recurrence, cells and packed lerps as march_sum, so the integrals are
// bitwise those of fp_forward_kernel) through the slab, reading the quads of
// a sample from the stage, or from global memory when the cell lies outside
// the box (rounding at its edge, or a bundle wider than the box), then meets
// the others at a barrier before the stage is refilled.  Waits on the copies
// are bounded: a timeout sets *error and the rays finish on global loads.

constexpr int kTmaO = 12;  // box cells across the bundle's main axis
constexpr int kTmaZ = 36;  // box quads along z (cells + 1)

struct TmaCorner {
    float o[3], d[3];  // voxel coordinates of the source and the ray direction per unit t
};

struct TmaSlab {
    int m0, o0, z0;  // padded index of the box origin along m, across, along z
};

// Box of slab id `sid` (padded m range [sid*L, sid*L + L)) from the corner
// rays' points on the slab's two faces, one cell of margin on each side.
template <int L>
__device__ __forceinline__ TmaSlab tma_slab_box(const TmaCorner* c, int m, int sid) {
    const int o = 1 - m;
    float omin = FLT_MAX, omax = -FLT_MAX, zmin = FLT_MAX, zmax = -FLT_MAX;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        const float plane = (float)(sid * L - 1 + f * L);  // voxel coordinate of the face
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float tau = (plane - c[k].o[m]) / c[k].d[m];
            const float oo = fmaf(tau, c[k].d[o], c[k].o[o]);
            const float zz = fmaf(tau, c[k].d[2], c[k].o[2]);
            omin = fminf(omin, oo);
            omax = fmaxf(omax, oo);
            zmin = fminf(zmin, zz);
            zmax = fmaxf(zmax, zz);
        }
    }
    TmaSlab b;
    b.m0 = sid * L;
    // padded index = floor + 1; one cell of margin below
    b.o0 = (int)floorf(omin);
    b.z0 = (int)floorf(zmin);
    // centre the box on the bundle when it is narrower than the box
    const int o_need = (int)floorf(omax) + 2 - b.o0, z_need = (int)floorf(zmax) + 3 - b.z0;
    if (o_need < kTmaO) b.o0 -= (kTmaO - o_need) / 2;
    if (z_need < kTmaZ) b.z0 -= (kTmaZ - z_need) / 2;
    return b;
}

template <int L>
__device__ __forceinline__ void tma_issue_slab(const TmaCorner* c, int m, int sid, int stage,
                                               TmaSlab* s_box_origin, ulonglong2* s_box,
                                               uint64_t* s_full, const CUtensorMap* map_x,
                                               const CUtensorMap* map_y) {
    constexpr uint32_t kBytes = (uint32_t)(L * kTmaO * kTmaZ * 16);
    const TmaSlab b = tma_slab_box<L>(c, m, sid);
    s_box_origin[stage] = b;
    const uint32_t bar = tma_smem_u32(&s_full[stage]);
    const uint32_t dst = tma_smem_u32(s_box + (size_t)stage * L * kTmaO * kTmaZ);
    tma_expect_tx(bar, kBytes);
    // x coordinate = 4 floats per quad: a multiple of 16 bytes for every z0
    if (m == 0) tma_load_3d(dst, map_x, 4 * b.z0, b.m0, b.o0, bar);
    else tma_load_3d(dst, map_y, 4 * b.z0, b.o0, b.m0, bar);
}

// Samples of one ray while their cell lies in the slab [m_lo, m_hi) (padded m
// index); returns with t at the first sample beyond it.
template <int L, bool CLAMP, bool DIV, bool OFF>
__device__ __forceinline__ void tma_march_slab(const RaySetup& r, const ViewGeo& vg, const FpArgs& p,
                                               const XYPacks& k, int m, int dir, int m_lo, int m_hi,
                                               const TmaSlab& b, const ulonglong2* __restrict__ box,
                                               bool use_box, int nmax, float& t, int& n,
                                               float& acc) {
    const ulonglong2* __restrict__ Q = reinterpret_cast<const ulonglong2*>(p.quads);
#pragma unroll 1
    for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
        const Cell c = sample_cell<CLAMP, DIV, OFF, true>(t, r, vg, p, k);
        const int px = (int)(c.bx - kFloorMagicBits) + 1, py = (int)(c.by - kFloorMagicBits) + 1;
        const int pz = (int)(c.bz - kFloorMagicBits) + 1;
        const int pm = m == 0 ? px : py, po = m == 0 ? py : px;
        if (dir > 0 ? pm >= m_hi : pm < m_lo) break;
        const int dm = pm - b.m0, dox = po - b.o0, dz = pz - b.z0;
        ulonglong2 q0, q1;
        if (use_box && (unsigned)dm < (unsigned)L && (unsigned)dox < (unsigned)kTmaO &&
            (unsigned)dz < (unsigned)(kTmaZ - 1)) {
            const int idx = (m == 0 ? (dox * L + dm) : (dm * kTmaO + dox)) * kTmaZ + dz;
            q0 = box[idx];
            q1 = box[idx + 1];
        } else {
            const uint32_t qi = quad_index(c, p);
            q0 = __ldg(Q + qi);
            q1 = __ldg(Q + qi + 1);
        }
        const f32x2 wx = pack2(c.fx, c.fx);
        const f32x2 e0 = lerp2(q0.x, q0.y, wx);
        const f32x2 e1 = lerp2(q1.x, q1.y, wx);
        const float2 e = unpack2(lerp2(e0, e1, pack2(c.fz, c.fz)));
        acc += lerpf(e.x, e.y, c.fy);
    }
}

template <int L, bool DIV, bool OFF>
__global__ void __launch_bounds__(256, 4) fp_forward_tma_kernel(FpArgs p,
                                                             const __grid_constant__ CUtensorMap map_x,
                                                             const __grid_constant__ CUtensorMap map_y,
                                                             int* error) {
    extern __shared__ __align__(128) ulonglong2 s_box[];  // two stages of L x kTmaO x kTmaZ quads
    __shared__ ViewGeo s_view;
    __shared__ __align__(8) uint64_t s_full[2];
    __shared__ TmaSlab s_origin[2];
    __shared__ TmaCorner s_corner[4];
    __shared__ int s_pm[2];
    __shared__ int s_issued[2];  // copies issued on each stage
    __shared__ int s_abort;
    constexpr int TU = 8;
    constexpr int kBoxQuads = L * kTmaO * kTmaZ;
    const int tiles_u = (p.U + TU - 1) / TU;
    const TileCoord tc = tile_coord(p, tiles_u);
    if (threadIdx.x == 0) {
        load_view(p.g, tc.a, s_view);
        tma_mbar_init(tma_smem_u32(&s_full[0]), 1);
        tma_mbar_init(tma_smem_u32(&s_full[1]), 1);
        tma_fence_init();
        s_pm[0] = INT_MAX;
        s_pm[1] = INT_MIN;
        s_issued[0] = s_issued[1] = 0;
        s_abort = 0;
    }
    __syncthreads();
    const ViewGeo vg = s_view;
    int u, v;
    tile_ray<TU>(tc, u, v);
    const bool in_range = u < p.U && v < p.V;
    const int uc = min(u, p.U - 1), vc = min(v, p.V - 1);
    const RaySetup r = setup_ray(vg, uc, vc, p);
    // main axis and direction of the bundle, from its central ray (the same
    // for every thread)
    const RaySetup rc = setup_ray(vg, min(tc.tu * TU + TU / 2, p.U - 1),
                                  min(tc.tv * 32 + 16, p.V - 1), p);
    const int m = fabsf(rc.dx) >= fabsf(rc.dy) ? 0 : 1;
    const int dir = (m == 0 ? rc.dx : rc.dy) >= 0.0f ? 1 : -1;
    const int n_m = m == 0 ? p.W : p.H;
    const float half_m = n_m * 0.5f;
    const float off_m = m == 0 ? p.off_x : p.off_y;
    const bool active = in_range && r.ok && r.hit;
    if (active) {
        // padded m index range of the ray's samples: between its box entry
        // and exit points, clamped to the padded volume
        const float om = m == 0 ? vg.ox : vg.oy, dm = m == 0 ? r.dx : r.dy;
        const float a = to_voxel<DIV, OFF>(fmaf(r.tmin, dm, om), off_m, p.voxel_size, p.inv_voxel,
                                           half_m);
        const float bb = to_voxel<DIV, OFF>(fmaf(r.tmax, dm, om), off_m, p.voxel_size, p.inv_voxel,
                                            half_m);
        const float lo = fminf(fmaxf(fminf(a, bb), -1.0f), (float)(n_m - 1));
        const float hi = fminf(fmaxf(fmaxf(a, bb), -1.0f), (float)(n_m - 1));
        atomicMin(&s_pm[0], (int)floorf(lo) + 1 - 1);  // one index of margin
        atomicMax(&s_pm[1], (int)floorf(hi) + 1 + 1);
    }
    // corner rays: warps 0 and 7, lanes 0 and 31
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if ((warp == 0 || warp == 7) && (lane == 0 || lane == 31)) {
        const int ci = (warp == 7 ? 2 : 0) + (lane == 31 ? 1 : 0);
        TmaCorner cr;
        const float ox = to_voxel<DIV, OFF>(vg.ox, p.off_x, p.voxel_size, p.inv_voxel, p.W * 0.5f);
        const float oy = to_voxel<DIV, OFF>(vg.oy, p.off_y, p.voxel_size, p.inv_voxel, p.H * 0.5f);
        const float oz = to_voxel<DIV, OFF>(vg.oz, p.off_z, p.voxel_size, p.inv_voxel, p.D * 0.5f);
        cr.o[0] = ox;
        cr.o[1] = oy;
        cr.o[2] = oz;
        cr.d[0] = r.dx / p.voxel_size;
        cr.d[1] = r.dy / p.voxel_size;
        cr.d[2] = r.dz / p.voxel_size;
        s_corner[ci] = cr;
    }
    __syncthreads();
    int pm_min = max(s_pm[0], 0), pm_max = min(s_pm[1], n_m);
    const int s_first = (dir > 0 ? pm_min : pm_max) / L;
    const int n_slabs = pm_min <= pm_max ? pm_max / L - pm_min / L + 1 : 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2 && i < n_slabs; ++i) {
            tma_issue_slab<L>(s_corner, m, s_first + dir * i, i, s_origin, s_box, s_full, &map_x,
                              &map_y);
            s_issued[i] += 1;
        }
    }
    __syncthreads();
    const XYPacks k = make_xy_packs(r, vg, p);
    const bool inside = active ? ray_inside_pad<DIV>(r, vg, p) : true;
    const int nmax = active ? step_bound(r, p.step_size) : 0;
    float t = r.tmin, acc = 0.0f;
    int n = 0;
    for (int i = 0; i < n_slabs; ++i) {
        const int stage = i & 1;
        const int sid = s_first + dir * i;
        // after an abort no further copies are issued: no wait, global loads
        bool have = false;
        if (!s_abort) {
            have = tma_wait(tma_smem_u32(&s_full[stage]), (uint32_t)((i >> 1) & 1));
            if (!have) {
                s_abort = 1;
                if (error) atomicExch(error, 1);
            }
        }
        if (active) {
            const TmaSlab b = s_origin[stage];
            const ulonglong2* box = s_box + (size_t)stage * kBoxQuads;
            const int m_lo = sid * L, m_hi = sid * L + L;
            if (inside)
                tma_march_slab<L, false, DIV, OFF>(r, vg, p, k, m, dir, m_lo, m_hi, b, box, have,
                                                   nmax, t, n, acc);
            else
                tma_march_slab<L, true, DIV, OFF>(r, vg, p, k, m, dir, m_lo, m_hi, b, box, have,
                                                  nmax, t, n, acc);
        }
        __syncthreads();  // every thread is done with this stage
        if (threadIdx.x == 0 && i + 2 < n_slabs && !s_abort) {
            tma_issue_slab<L>(s_corner, m, s_first + dir * (i + 2), stage, s_origin, s_box, s_full,
                              &map_x, &map_y);
            s_issued[stage] += 1;
        }
        __syncthreads();  // s_abort and the next stage's origin as thread 0 left them
    }
    if (threadIdx.x == 0) {
        // no copy may still write into this CTA's shared memory when it exits:
        // wait (bounded) for the last copy of each stage; returns at once for
        // copies already waited for
        for (int st = 0; st < 2; ++st)
            if (s_issued[st] > 0)
                tma_wait(tma_smem_u32(&s_full[st]), (uint32_t)((s_issued[st] - 1) & 1));
    }
    if (active) {
        // samples past the last slab (none unless rounding put a cell beyond
        // the bundle's range): global loads
        if (inside)
            tma_march_slab<L, false, DIV, OFF>(r, vg, p, k, m, dir, dir > 0 ? 0 : INT_MIN,
                                               dir > 0 ? INT_MAX : INT_MAX, TmaSlab{0, 0, 0},
                                               nullptr, false, nmax, t, n, acc);
        else
            tma_march_slab<L, true, DIV, OFF>(r, vg, p, k, m, dir, dir > 0 ? 0 : INT_MIN,
                                              dir > 0 ? INT_MAX : INT_MAX, TmaSlab{0, 0, 0},
                                              nullptr, false, nmax, t, n, acc);
    }
    if (in_range) p.projections[((long long)tc.a * p.U + u) * p.V + v] = active ? acc * p.step_size : 0.0f;
}

// Sample counts under the same FP32 rule (measurement support).
__global__ void __launch_bounds__(256) fp_count_kernel(FpArgs p, int64_t* __restrict__ counts) {
    constexpr int TU = 8, TV = 32;
    __shared__ ViewGeo s_view;
    const int tiles_u = (p.U + TU - 1) / TU;
    const TileCoord tc = tile_coord(p, tiles_u);
    if (threadIdx.x == 0) load_view(p.g, tc.a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    const int u = tc.tu * TU + (threadIdx.x >> 5);
    const int v = tc.tv * TV + (threadIdx.x & 31);
    if (u >= p.U || v >= p.V) return;
    const RaySetup r = setup_ray(vg, u, v, p);
    long long n = 0;
    if (r.ok && r.hit) {
        const int nmax = step_bound(r, p.step_size);
        for (float t = r.tmin; t <= r.tmax && n < nmax; t += p.step_size) ++n;
    }
    counts[((long long)tc.a * p.U + u) * p.V + v] = n;
}

// ---------------------------------------------------------------------------
// Backward kernel: volume adjoint (optional) + per-ray geometry terms
// ---------------------------------------------------------------------------

struct RayGrad {
    // s1 = sum of the voxel-unit spatial gradient g over the samples,
    // s2 = sum of g * (t - t_min).
    float s1x, s1y, s1z, s2x, s2y, s2z;
};

// GRADVOL: also scatter the adjoint of every sample into p.grad_pad, a
// cell-major buffer of 16-byte level records R[(cy*(W+1) + cx)*(D+2) + cz]
// (cells at padded index floor+1): record c holds the weights of the four
// corners (cz, cy+dy, cx+dx) of its z level at dy*2 + dx, so a sample adds
// its z level to its cell's record and its z+1 level to the next record;
// fold_record_gradient_kernel then sums the records onto the voxels.  A
// lane's consecutive samples of one cell are first added in registers.
template <bool CLAMP, bool GRADVOL>
__device__ __forceinline__ RayGrad march_grad(const RaySetup& r, const ViewGeo& vg,
                                              const FpArgs& p, float gs) {
    const ulonglong2* __restrict__ Q = reinterpret_cast<const ulonglong2*>(p.quads);
    const XYPacks k = make_xy_packs(r, vg, p);
    RayGrad rg{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int nmax = step_bound(r, p.step_size);
    // this lane's pending level records (cell run_ci: its z level and z+1
    // level), flushed when the ray leaves the cell
    const f32x2 zero = pack2(0.0f, 0.0f);
    uint32_t run_ci = 0u;
    bool run_have = false;
    f32x2 run_lo[2] = {zero, zero}, run_hi[2] = {zero, zero};
    float t = r.tmin;
    int n = 0;
#pragma unroll 1
    for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
        const Cell c = sample_cell<CLAMP, false, true, false>(t, r, vg, p, k);
        const uint32_t qi = quad_index(c, p);
        const ulonglong2 q0 = __ldg(Q + qi);
        const ulonglong2 q1 = __ldg(Q + qi + 1);
        // d/dx, d/dy, d/dz of the trilinear interpolant (voxel units), from
        // packed (y0, y1) pairs: .x of a quad is x0, .y is x1
        const f32x2 wx = pack2(c.fx, c.fx), wz = pack2(c.fz, c.fz);
        const f32x2 d0 = sub2(q0.y, q0.x), d1 = sub2(q1.y, q1.x);  // x1 - x0
        const f32x2 e0 = fma2(wx, d0, q0.x), e1 = fma2(wx, d1, q1.x);
        const f32x2 ez = sub2(e1, e0);
        const float2 e = unpack2(fma2(wz, ez, e0));
        const float2 dx = unpack2(fma2(wz, sub2(d1, d0), d0));
        const float2 dz = unpack2(ez);
        const float gx = lerpf(dx.x, dx.y, c.fy);
        const float gy = e.y - e.x;
        const float gz = lerpf(dz.x, dz.y, c.fy);
        const float tau = t - r.tmin;
        rg.s1x += gx;
        rg.s1y += gy;
        rg.s1z += gz;
        rg.s2x = fmaf(gx, tau, rg.s2x);
        rg.s2y = fmaf(gy, tau, rg.s2y);
        rg.s2z = fmaf(gz, tau, rg.s2z);
        if (GRADVOL) {
            // adjoint of the trilinear sample (fp.cu:231-240) into the level records
            const float mx = 1.0f - c.fx, my = 1.0f - c.fy, mz = 1.0f - c.fz;
            const float gy0 = gs * my, gy1 = gs * c.fy;
            // (x, y) corner columns 00, 10, 01, 11 at the cell's z (lo) and z+1
            // (hi) as packed pairs: w0 = (w00, w01), w1 = (w10, w11), the
            // products lane by lane those of the scalar form
            const f32x2 wxs = pack2(mx, c.fx);
            const f32x2 w0 = mul2(pack2(gy0, gy0), wxs), w1 = mul2(pack2(gy1, gy1), wxs);
            const f32x2 zl = pack2(mz, mz), zh = pack2(c.fz, c.fz);
            f32x2 lo2[2] = {mul2(w0, zl), mul2(w1, zl)};
            f32x2 hi2[2] = {mul2(w0, zh), mul2(w1, zh)};
            const uint32_t gi = c.bz + c.bx * p.gz_x + c.by * p.gz_y + p.gz_bias;
            {
                // Consecutive samples of the ray mostly share a cell: add them
                // in registers and emit a cell's two level records when the
                // ray moves on.  A move to the cell above (below) in z shares a
                // level, which stays pending.  Branch-free: predicated
                // reductions of the pending records, then selects.
                const int d = (int)(gi - run_ci);
                const bool same = run_have && d == 0, up = run_have && d == 1,
                           down = run_have && d == -1;
                float* o = p.grad_pad + 4ull * run_ci;
                const float2 a0 = unpack2(run_lo[0]), a1 = unpack2(run_lo[1]);
                const float2 b0 = unpack2(run_hi[0]), b1 = unpack2(run_hi[1]);
                red_add4_global_if(run_have && !same && !down, o, a0.x, a0.y, a1.x, a1.y);
                red_add4_global_if(run_have && !same && !up, o + 4, b0.x, b0.y, b1.x, b1.y);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const f32x2 base_lo = same ? run_lo[j] : up ? run_hi[j] : zero;
                    const f32x2 base_hi = same ? run_hi[j] : down ? run_lo[j] : zero;
                    run_lo[j] = add2(base_lo, lo2[j]);
                    run_hi[j] = add2(base_hi, hi2[j]);
                }
                run_ci = gi;
                run_have = true;
            }
        }
    }
    if (GRADVOL && run_have) {
        float* o = p.grad_pad + 4ull * run_ci;
        const float2 a0 = unpack2(run_lo[0]), a1 = unpack2(run_lo[1]);
        const float2 b0 = unpack2(run_hi[0]), b1 = unpack2(run_hi[1]);
        red_add4_global(o, a0.x, a0.y, a1.x, a1.y);
        red_add4_global(o + 4, b0.x, b0.y, b1.x, b1.y);
    }
    return rg;
}

// The eight per-view geometry terms of a ray that hits the volume, from its
// march sums and gs = dL/dp * step.
__device__ __forceinline__ void ray_geometry_terms(const FpArgs& p, const ViewGeo& vg,
                                                   const RaySetup& r, int u, const RayGrad& rg,
                                                   float gs, float (&terms)[8]) {
    // fp.cu:441-467 give, with G = gs/voxel,
    //   grad_origin_direct = G*s1 - (G*(s1.d)/d_e) e_e
    //   grad_direction     = G*sum g*t - (G*(s1.d) t_min/d_e) e_e
    // (e = entry axis).  Writing sum g*t = s2 + t_min*s1 and
    //   q = s1 - ((s1.d)/d_e) e_e   (so q.d = 0)
    // gives grad_origin_direct = G*q and grad_direction = G*(s2 + t_min*q):
    // the same values without the large t_min*s1 terms that cancel.
    // (the multiply-adds are explicit, as in the ray set-up, so that every
    // kernel that inlines this produces bitwise the same terms)
    float qx = rg.s1x, qy = rg.s1y, qz = rg.s1z;
    if (r.entry_axis == 0) qx = -fmaf(rg.s1y, r.dy, __fmul_rn(rg.s1z, r.dz)) / r.dx;
    else if (r.entry_axis == 1) qy = -fmaf(rg.s1x, r.dx, __fmul_rn(rg.s1z, r.dz)) / r.dy;
    else if (r.entry_axis == 2) qz = -fmaf(rg.s1x, r.dx, __fmul_rn(rg.s1y, r.dy)) / r.dz;
    const float G = gs * p.inv_voxel;
    const float godx = G * qx, gody = G * qy, godz = G * qz;
    // fp.cu:470-486: chain through direction = normalize(target - origin);
    // q is orthogonal to d, so only s2 loses its component along d.
    const float ds2 = fmaf(r.dz, rg.s2z, fmaf(r.dx, rg.s2x, __fmul_rn(r.dy, rg.s2y)));
    const float k = G / r.len;
    const float grx = k * fmaf(r.tmin, qx, fmaf(-r.dx, ds2, rg.s2x));
    const float gry = k * fmaf(r.tmin, qy, fmaf(-r.dy, ds2, rg.s2y));
    const float grz = k * fmaf(r.tmin, qz, fmaf(-r.dz, ds2, rg.s2z));
    const float gox = godx - grx, goy = gody - gry, goz = godz - grz;
    // fp.cu:488-527: per-view geometry terms.
    const float u_phys = (u - vg.u0) * p.pixel_size;
    const float dOx = -vg.sod * vg.c, dOy = -vg.sod * vg.s;
    const float dTx = fmaf(-u_phys, vg.s, -__fmul_rn(vg.dn, vg.c));
    const float dTy = fmaf(u_phys, vg.c, -__fmul_rn(vg.dn, vg.s));
    terms[0] = fmaf(gry, dTy, fmaf(grx, dTx, fmaf(goy, dOy, __fmul_rn(gox, dOx))));
    terms[1] = fmaf(grx, vg.s, -__fmul_rn(gry, vg.c));
    terms[2] = fmaf(goy + gry, vg.c, -__fmul_rn(gox + grx, vg.s));
    terms[3] = -p.pixel_size * fmaf(grx, vg.c, __fmul_rn(gry, vg.s));
    terms[4] = -p.pixel_size * grz;
    terms[5] = gox;
    terms[6] = goy;
    terms[7] = goz;
}

// The eight per-view geometry terms of one ray (zero for rays outside the
// detector, missing the volume or with a zero upstream gradient); with
// GRADVOL (march_grad) the ray's adjoint samples go into p.grad_pad.
template <bool GRADVOL>
__device__ __forceinline__ void backward_ray(const FpArgs& p, const ViewGeo& vg, int a, int u,
                                             int v, float (&terms)[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) terms[k] = 0.0f;
    const bool in_range = u < p.U && v < p.V;
    const float grad_out =
        in_range ? p.grad_projections[((long long)a * p.U + u) * p.V + v] : 0.0f;
    // fp.cu:381 -- rays with a zero upstream gradient contribute nothing.
    if (in_range && grad_out != 0.0f) {
        const RaySetup r = setup_ray(vg, u, v, p);
        if (r.ok && r.hit) {
            const float gs = grad_out * p.step_size;
            const RayGrad rg = ray_inside_pad<false>(r, vg, p)
                                   ? march_grad<false, GRADVOL>(r, vg, p, gs)
                                   : march_grad<true, GRADVOL>(r, vg, p, gs);
            ray_geometry_terms(p, vg, r, u, rg, gs, terms);
        }
    }
}

// Fixed-order FP64 sum of the eight terms over the 256 threads of the CTA,
// written to partials[(a * tiles + tile) * 8 + k].
__device__ __forceinline__ void reduce_terms_to_partials(const float (&terms)[8],
                                                         double (&s_red)[8][8],
                                                         double* __restrict__ out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const double w = warp_sum((double)terms[k]);
        if (lane == 0) s_red[warp][k] = w;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) acc += s_red[w][threadIdx.x];
        out[threadIdx.x] = acc;
    }
}

template <int TU, bool GRADVOL>
__global__ void __launch_bounds__(256) fp_backward_kernel(FpArgs p) {
    constexpr int TV = 256 / TU;
    __shared__ ViewGeo s_view;
    __shared__ double s_red[8][8];
    const int tiles_u = (p.U + TU - 1) / TU;
    const int tiles = tiles_u * ((p.V + TV - 1) / TV);
    const TileCoord tc = tile_coord(p, tiles_u);
    const int a = tc.a;
    const int tile = tc.tv * tiles_u + tc.tu;
    if (threadIdx.x == 0) load_view(p.g, a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    int u, v;
    tile_ray<TU>(tc, u, v);
    float terms[8];
    backward_ray<GRADVOL>(p, vg, a, u, v, terms);
    reduce_terms_to_partials(terms, s_red, p.partials + ((long long)a * tiles + tile) * 8);
}

// ---------------------------------------------------------------------------
// Fused projection -> masked MSE -> geometry gradients (calibration step)
// ---------------------------------------------------------------------------

struct RayValueGrad {
    float sum;  // sum of the trilinear samples (the forward kernel's arithmetic)
    RayGrad g;  // s1, s2 of march_grad
};

// One march that yields both the line-integral sum (bitwise the forward
// kernel's: same positions, same packed lerps) and the spatial-gradient sums
// of the backward.  No scatter: the volume is not differentiated here.
template <bool CLAMP, bool DIV, bool OFF, bool GUARD = true>
__device__ __forceinline__ RayValueGrad march_value_grad(const RaySetup& r, const ViewGeo& vg,
                                                         const FpArgs& p) {
    const ulonglong2* __restrict__ Q = reinterpret_cast<const ulonglong2*>(p.quads);
    const XYPacks k = make_xy_packs(r, vg, p);
    RayValueGrad out{0.0f, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
    const int nmax = step_bound(r, p.step_size);
    float t = r.tmin;
    int n = 0;
#pragma unroll 1
    for (; t <= r.tmax && (!GUARD || n < nmax); t += p.step_size, n += GUARD ? 1 : 0) {
        const Cell c = sample_cell<CLAMP, DIV, OFF, false>(t, r, vg, p, k);
        const uint32_t qi = quad_index(c, p);
        const ulonglong2 q0 = __ldg(Q + qi);
        const ulonglong2 q1 = __ldg(Q + qi + 1);
        // value: exactly the forward kernel's packed lerps (lerp2(a, b, w) =
        // fma2(w, b - a, a)), keeping the intermediate pairs
        const f32x2 wx = pack2(c.fx, c.fx), wz = pack2(c.fz, c.fz);
        const f32x2 d0 = sub2(q0.y, q0.x);  // x1 - x0 at (y0, y1), z0
        const f32x2 d1 = sub2(q1.y, q1.x);  // x1 - x0 at (y0, y1), z1
        const f32x2 e0 = fma2(wx, d0, q0.x);
        const f32x2 e1 = fma2(wx, d1, q1.x);
        const f32x2 ez = sub2(e1, e0);
        const float2 e = unpack2(fma2(wz, ez, e0));
        out.sum += lerpf(e.x, e.y, c.fy);
        // spatial gradient from the same pairs (the trilinear interpolant is
        // linear along each axis): d/dx = lerp_y(lerp_z(x1 - x0)),
        // d/dy = Y1 - Y0, d/dz = lerp_y(lerp_x(z1) - lerp_x(z0))
        const float2 dx = unpack2(fma2(wz, sub2(d1, d0), d0));
        const float2 dz = unpack2(ez);
        const float gx = lerpf(dx.x, dx.y, c.fy);
        const float gy = e.y - e.x;
        const float gz = lerpf(dz.x, dz.y, c.fy);
        const float tau = t - r.tmin;
        out.g.s1x += gx;
        out.g.s1y += gy;
        out.g.s1z += gz;
        out.g.s2x = fmaf(gx, tau, out.g.s2x);
        out.g.s2y = fmaf(gy, tau, out.g.s2y);
        out.g.s2z = fmaf(gz, tau, out.g.s2z);
    }
    return out;
}

// Per ray: p = projection, L_ray = mask * (p - measured)^2, dL/dp = 2 * scale *
// mask * (p - measured); the geometry terms of the backward with that upstream
// gradient.  Per CTA: FP64 fixed-order sums of the eight terms (partials) and
// of L_ray (loss_partials).
template <int TU, bool DIV, bool OFF>
__global__ void __launch_bounds__(256) fp_mse_grad_kernel(FpArgs p, const float* __restrict__ measured,
                                                          const float* __restrict__ mask, float scale,
                                                          double* __restrict__ loss_partials) {
    constexpr int TV = 256 / TU;
    __shared__ ViewGeo s_view;
    __shared__ double s_red[8][8];
    __shared__ double s_loss[8];
    const int tiles_u = (p.U + TU - 1) / TU;
    const int tiles = tiles_u * ((p.V + TV - 1) / TV);
    const TileCoord tc = tile_coord(p, tiles_u);
    const int a = tc.a;
    const int tile = tc.tv * tiles_u + tc.tu;
    if (threadIdx.x == 0) load_view(p.g, a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    int u, v;
    tile_ray<TU>(tc, u, v);
    float terms[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float lray = 0.0f;
    if (u < p.U && v < p.V) {
        const RaySetup r = setup_ray(vg, u, v, p);
        RayValueGrad m{0.0f, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
        const bool hit = r.ok && r.hit;
        if (hit) {
            const bool inside = ray_inside_pad<DIV>(r, vg, p);
            if (steps_advance(r, p.step_size))
                m = inside ? march_value_grad<false, DIV, OFF, false>(r, vg, p)
                           : march_value_grad<true, DIV, OFF, false>(r, vg, p);
            else
                m = inside ? march_value_grad<false, DIV, OFF>(r, vg, p)
                           : march_value_grad<true, DIV, OFF>(r, vg, p);
        }
        const float proj = m.sum * p.step_size;
        const long long idx = ((long long)a * p.U + u) * p.V + v;
        if (p.projections) p.projections[idx] = proj;
        const float w = mask ? mask[idx] : 1.0f;
        const float diff = proj - measured[idx];
        lray = w * diff * diff;
        const float g = 2.0f * scale * w * diff;
        if (hit && g != 0.0f) ray_geometry_terms(p, vg, r, u, m.g, g * p.step_size, terms);
    }
    reduce_terms_to_partials(terms, s_red, p.partials + ((long long)a * tiles + tile) * 8);
    const double l = warp_sum((double)lray);
    if ((threadIdx.x & 31) == 0) s_loss[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) acc += s_loss[w];
        loss_partials[(long long)a * tiles + tile] = acc;
    }
}

// Fixed-order sum of n doubles by one block of 256 threads: out[0] = scale * sum.
__global__ void __launch_bounds__(256) sum_partials_kernel(const double* __restrict__ x, long long n,
                                                           double scale, double* __restrict__ out) {
    __shared__ double s[8];
    double acc = 0.0;
    for (long long i = threadIdx.x; i < n; i += 256) acc += x[i];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += s[w];
        out[0] = scale * t;
    }
}

// Per-view sum of the CTA partials, warp k owning gradient k (fixed order).
__global__ void __launch_bounds__(256) reduce_view_partials_kernel(const double* __restrict__ partials,
                                                                   int tiles, GeometryGrad out) {
    const int a = blockIdx.x;
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int i = lane; i < tiles; i += 32) acc += partials[((long long)a * tiles + i) * 8 + k];
    acc = warp_sum(acc);
    if (lane == 0) out.g[k][a] = (float)acc;
}

// Volume gradient from the level records R[((cy*(W+1) + cx)*(D+2) + cz)*4 + k]
// (march_grad; cells at padded index floor+1 in [0, n]): a padded corner P
// gets entry k = dy*2 + dx of record P - (0, dy, dx) for every record in range,
// and padded corners fold onto the clamped voxels (index 0 onto 0, n+1 onto
// n-1, as the clamped neighbours of fp.cu:200-213 sample them).
__device__ __forceinline__ float fold_record_voxel(const float* __restrict__ O, int D, int H, int W,
                                                   long long i) {
    const long long CZ = D + 2, CX = W + 1;
    const int x = (int)(i % W);
    const long long r = i / W;
    const int y = (int)(r % H);
    const int z = (int)(r / H);
    int xs[3], ys[3], zs[3];
    int nx = 0, ny = 0, nz = 0;
    xs[nx++] = x + 1;
    if (x == 0) xs[nx++] = 0;
    if (x == W - 1) xs[nx++] = W + 1;
    ys[ny++] = y + 1;
    if (y == 0) ys[ny++] = 0;
    if (y == H - 1) ys[ny++] = H + 1;
    zs[nz++] = z + 1;
    if (z == 0) zs[nz++] = 0;
    if (z == D - 1) zs[nz++] = D + 1;
    float acc = 0.0f;
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix)
            for (int iz = 0; iz < nz; ++iz)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int dy = k >> 1, dx = k & 1;
                    const int cz = zs[iz], cy = ys[iy] - dy, cx = xs[ix] - dx;
                    if (cy < 0 || cy > H || cx < 0 || cx > W) continue;
                    acc += O[((cy * CX + cx) * CZ + cz) * 4 + k];
                }
    return acc;
}

__global__ void fold_record_gradient_kernel(const float* __restrict__ O, int D, int H, int W,
                                            float* __restrict__ grad) {
    const long long total = (long long)D * H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        grad[i] = fold_record_voxel(O, D, H, W, i);
}

// ---------------------------------------------------------------------------
// Batched launches: many instances of uneven D/H/W, A, U, V in one launch.
//
// A work item is one CTA tile of one instance, numbered instance by instance
// and inside an instance in the single-instance order (u tile fastest, then
// view, then row band).  The forward and backward kernels are persistent:
// each CTA takes the next item from a global counter, loads the instance's
// arguments and the view geometry into shared memory and runs the same ray
// code as the single-instance kernels, with the tile shape and the division /
// offset variants its instance was planned with.  Items are taken in order,
// so the CTAs in flight work on one or two instances at a time (their
// volumes stay in L2), and a small instance fills the SMs that a large one
// leaves idle at its end.  The per-instance set-up kernels (quads, partial
// reductions, gradient folds) are flattened over instances the same way.
// ---------------------------------------------------------------------------

// Largest i with starts[i] <= x (starts nondecreasing, starts[0] = 0).
__device__ __forceinline__ int find_instance(const long long* __restrict__ starts, int n,
                                             long long x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(starts + mid) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ TileCoord item_coord(long long local, int tiles_u, int A) {
    TileCoord tc;
    tc.tu = (int)(local % tiles_u);
    const long long r = local / tiles_u;
    tc.a = (int)(r % A);
    tc.tv = (int)(r / A);
    return tc;
}

__global__ void __launch_bounds__(256) batch_quads_kernel(BatchTables t) {
    __shared__ float4 tile[32][33];
    const int i = find_instance(t.quad_block, t.n, blockIdx.x);
    const BatchInstance& in = t.inst[i];
    const long long b = blockIdx.x - t.quad_block[i];
    quads_tile(in.volume, in.p.D, in.p.H, in.p.W, const_cast<float4*>(in.p.quads),
               (int)(b % in.quad_gx), (int)(b / in.quad_gx), tile);
}

// Thread 0 takes the next item of the queue and stages its instance and view.
__device__ __forceinline__ bool next_item(const BatchTables& t, const long long* __restrict__ starts,
                                          unsigned long long* counter, bool backward,
                                          FpArgs& s_p, ViewGeo& s_view, TileCoord& s_tc,
                                          int& s_tu, int& s_flags, int& s_tile,
                                          long long& s_item) {
    if (threadIdx.x == 0) {
        const long long total = starts[t.n];
        const long long item = (long long)atomicAdd(counter, 1ULL);
        s_item = item;
        if (item < total) {
            const int i = find_instance(starts, t.n, item);
            const BatchInstance& in = t.inst[i];
            const int tu = backward ? in.tile_bwd : in.tile_fwd;
            const int tiles_u = (in.p.U + tu - 1) / tu;
            const TileCoord tc = item_coord(item - starts[i], tiles_u, in.p.A);
            s_p = in.p;
            s_tu = tu;
            s_flags = in.flags;
            s_tc = tc;
            s_tile = tc.tv * tiles_u + tc.tu;
            load_view(in.p.g, tc.a, s_view);
        }
    }
    __syncthreads();
    return s_item < starts[t.n];
}

template <int TU>
__device__ __forceinline__ void forward_item(const FpArgs& p, const ViewGeo& vg,
                                             const TileCoord& tc, int flags) {
    int u, v;
    tile_ray<TU>(tc, u, v);
    if (u >= p.U || v >= p.V) return;
    switch (flags & (kBatchDiv | kBatchOff)) {
        case 0: forward_ray<false, false>(p, vg, tc.a, u, v); break;
        case kBatchOff: forward_ray<false, true>(p, vg, tc.a, u, v); break;
        case kBatchDiv: forward_ray<true, false>(p, vg, tc.a, u, v); break;
        default: forward_ray<true, true>(p, vg, tc.a, u, v); break;
    }
}

__global__ void __launch_bounds__(256, 6) batch_forward_kernel(BatchTables t) {
    __shared__ FpArgs s_p;
    __shared__ ViewGeo s_view;
    __shared__ TileCoord s_tc;
    __shared__ int s_tu, s_flags, s_tile;
    __shared__ long long s_item;
    while (next_item(t, t.item_fwd, t.counters, false, s_p, s_view, s_tc, s_tu, s_flags, s_tile,
                     s_item)) {
        const FpArgs p = s_p;
        const ViewGeo vg = s_view;
        const TileCoord tc = s_tc;
        switch (s_tu) {
            case 8: forward_item<8>(p, vg, tc, s_flags); break;
            case 4: forward_item<4>(p, vg, tc, s_flags); break;
            default: forward_item<2>(p, vg, tc, s_flags); break;
        }
        __syncthreads();  // the staged item is read by every thread before the next one
    }
}

template <int TU>
__device__ __forceinline__ void backward_item(const FpArgs& p, const ViewGeo& vg,
                                              const TileCoord& tc, float (&terms)[8]) {
    int u, v;
    tile_ray<TU>(tc, u, v);
    if (p.grad_pad) backward_ray<true>(p, vg, tc.a, u, v, terms);
    else backward_ray<false>(p, vg, tc.a, u, v, terms);
}

__global__ void __launch_bounds__(256, 4) batch_backward_kernel(BatchTables t) {
    __shared__ FpArgs s_p;
    __shared__ ViewGeo s_view;
    __shared__ TileCoord s_tc;
    __shared__ int s_tu, s_flags, s_tile;
    __shared__ long long s_item;
    __shared__ double s_red[8][8];
    while (next_item(t, t.item_bwd, t.counters + 1, true, s_p, s_view, s_tc, s_tu, s_flags,
                     s_tile, s_item)) {
        const FpArgs p = s_p;
        const ViewGeo vg = s_view;
        const TileCoord tc = s_tc;
        float terms[8];
        if (s_tu == 8) backward_item<8>(p, vg, tc, terms);
        else backward_item<4>(p, vg, tc, terms);
        const long long tiles = fp_tiles_per_view_dev(p.U, p.V, s_tu);
        reduce_terms_to_partials(terms, s_red, p.partials + ((long long)tc.a * tiles + s_tile) * 8);
        __syncthreads();
    }
}

// One block per view of every instance (the order of reduce_view_partials_kernel).
__global__ void __launch_bounds__(256) batch_reduce_kernel(BatchTables t) {
    const int i = find_instance(t.view, t.n, blockIdx.x);
    const BatchInstance& in = t.inst[i];
    const int a = (int)(blockIdx.x - t.view[i]);
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tiles = in.tiles_bwd;
    const double* __restrict__ partials = in.p.partials;
    double acc = 0.0;
    for (long long j = lane; j < tiles; j += 32) acc += partials[((long long)a * tiles + j) * 8 + k];
    acc = warp_sum(acc);
    if (lane == 0) in.gout.g[k][a] = (float)acc;
}

// kFoldChunk voxels of one instance per block.
__global__ void __launch_bounds__(256) batch_fold_kernel(BatchTables t) {
    const int i = find_instance(t.fold_block, t.n, blockIdx.x);
    const BatchInstance& in = t.inst[i];
    const long long total = (long long)in.p.D * in.p.H * in.p.W;
    const long long v0 = (blockIdx.x - t.fold_block[i]) * (long long)kFoldChunk;
    const long long v1 = v0 + kFoldChunk < total ? v0 + kFoldChunk : total;
    for (long long v = v0 + threadIdx.x; v < v1; v += blockDim.x)
        in.grad_volume[v] = fold_record_voxel(in.p.grad_pad, in.p.D, in.p.H, in.p.W, v);
}

// ---------------------------------------------------------------------------
// Launch configuration
// ---------------------------------------------------------------------------

namespace {

template <int TU, int UNROLL = 1>
int launch_forward_tu(const FpArgs& p, bool div, cudaStream_t s) {
    DGC_TRACE("fp_forward_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    const bool off = p.off_x != 0.0f || p.off_y != 0.0f || p.off_z != 0.0f;
    if (div) {
        if (off) fp_forward_kernel<TU, true, true, UNROLL><<<(unsigned)blocks, 256, 0, s>>>(p);
        else fp_forward_kernel<TU, true, false, UNROLL><<<(unsigned)blocks, 256, 0, s>>>(p);
    } else {
        if (off) fp_forward_kernel<TU, false, true, UNROLL><<<(unsigned)blocks, 256, 0, s>>>(p);
        else fp_forward_kernel<TU, false, false, UNROLL><<<(unsigned)blocks, 256, 0, s>>>(p);
    }
    DGC_LAUNCH_CHECK("fp_forward_kernel");
    return DGC_OK;
}

template <int TU>
int launch_backward_tu(const FpArgs& p, bool gradvol, cudaStream_t s) {
    DGC_TRACE(gradvol ? "fp_backward_kernel<gradvol>" : "fp_backward_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    if (gradvol) fp_backward_kernel<TU, true><<<(unsigned)blocks, 256, 0, s>>>(p);
    else fp_backward_kernel<TU, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fp_backward_kernel");
    return DGC_OK;
}

}  // namespace

size_t fp_record_buffer_floats(int D, int H, int W) {
    return 4 * (size_t)(D + 2) * (size_t)(H + 1) * (size_t)(W + 1);
}

int fp_fold_records(const float* records, int D, int H, int W, float* grad, cudaStream_t s) {
    DGC_TRACE("fold_record_gradient", s);
    const long long total = (long long)D * H * W;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    fold_record_gradient_kernel<<<blocks, 256, 0, s>>>(records, D, H, W, grad);
    DGC_LAUNCH_CHECK("fold_record_gradient");
    return DGC_OK;
}

long long fp_tiles_per_view(int U, int V, int tu) {
    const int tv = 256 / tu;
    return (long long)ceil_div(U, tu) * ceil_div(V, tv);
}

void fp_fill_layout(FpArgs& p) {
    // quads: Q[(yp*(W+1) + xp)*(D+2) + zp]; index of (z0+1, y0+1, x0+1) from
    // the biased floors bz, bx, by (modular 32-bit arithmetic)
    p.zq_x = (uint32_t)(p.D + 2);
    p.zq_y = (uint32_t)(p.W + 1) * (uint32_t)(p.D + 2);
    p.zq_bias = (1u + p.zq_x + p.zq_y) - kFloorMagicBits * (1u + p.zq_x + p.zq_y);
    // level records of the volume gradient: record index of padded cell
    // (floor+1) from the biased floors, R[(yp*(W+1) + xp)*(D+2) + zp]
    p.gz_x = (uint32_t)(p.D + 2);
    p.gz_y = (uint32_t)(p.W + 1) * (uint32_t)(p.D + 2);
    p.gz_bias = (1u + p.gz_x + p.gz_y) - kFloorMagicBits * (1u + p.gz_x + p.gz_y);
    p.inv_voxel = 1.0f / p.voxel_size;
}

namespace {

// Arm rules (what the autotuner chose per volume size): the first rule with
// D*H*W <= voxels_max applies; without one the L1 arm runs.
struct FpArmRule {
    long long voxels_max;
    int arm, slab, unroll, view_block;
};
std::mutex g_arm_mutex;
FpArmRule g_arm_rules[16];
int g_arm_count = 0;

template <int L, bool DIV, bool OFF>
int launch_tma_variant(const FpArgs& p, const CUtensorMap& mx, const CUtensorMap& my,
                       long long blocks, cudaStream_t s) {
    constexpr int smem = 2 * L * kTmaO * kTmaZ * 16;
    static std::atomic<unsigned long long> configured{0};
    const int rc = once_per_device(configured, []() -> int {
        DGC_CUDA(cudaFuncSetAttribute(fp_forward_tma_kernel<L, DIV, OFF>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        return DGC_OK;
    });
    if (rc != DGC_OK) return rc;
    fp_forward_tma_kernel<L, DIV, OFF><<<(unsigned)blocks, 256, smem, s>>>(p, mx, my, p.error);
    return DGC_OK;
}

// 3-D float map of the quad volume, innermost first: 4*(D+2) floats, W+1, H+1.
bool quad_volume_map(CUtensorMap* map, const FpArgs& p, int box_z, int box_x, int box_y) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)4 * (p.D + 2), (cuuint64_t)(p.W + 1),
                                (cuuint64_t)(p.H + 1)};
    const cuuint64_t strides[2] = {(cuuint64_t)16 * (p.D + 2),
                                   (cuuint64_t)16 * (p.D + 2) * (cuuint64_t)(p.W + 1)};
    const cuuint32_t box[3] = {(cuuint32_t)(4 * box_z), (cuuint32_t)box_x, (cuuint32_t)box_y};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float4*>(p.quads), dims, strides,
              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

template <int L>
int launch_forward_tma(const FpArgs& p, bool div, cudaStream_t s, bool* used) {
    *used = false;
    CUtensorMap mx, my;
    if (!quad_volume_map(&mx, p, kTmaZ, L, kTmaO) || !quad_volume_map(&my, p, kTmaZ, kTmaO, L))
        return DGC_OK;
    *used = true;
    DGC_TRACE("fp_forward_tma_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, 8) * (long long)p.A;
    const bool off = p.off_x != 0.0f || p.off_y != 0.0f || p.off_z != 0.0f;
    int rc;
    if (div) rc = off ? launch_tma_variant<L, true, true>(p, mx, my, blocks, s)
                      : launch_tma_variant<L, true, false>(p, mx, my, blocks, s);
    else rc = off ? launch_tma_variant<L, false, true>(p, mx, my, blocks, s)
                  : launch_tma_variant<L, false, false>(p, mx, my, blocks, s);
    if (rc != DGC_OK) return rc;
    DGC_LAUNCH_CHECK("fp_forward_tma_kernel");
    return DGC_OK;
}

}  // namespace

int fp_add_arm_rule(long long voxels_max, int arm, int slab, int unroll, int view_block) {
    if (voxels_max < 1 || arm < 0 || arm > 2 || (arm == 1 && slab != 2 && slab != 4) ||
        (unroll != 1 && unroll != 2) || (arm != 0 && unroll != 1) || view_block < 0 ||
        view_block > 65535)
        return -1;
    std::lock_guard<std::mutex> lock(g_arm_mutex);
    if (g_arm_count >= 16) return -2;
    g_arm_rules[g_arm_count++] =
        FpArmRule{voxels_max, arm, arm == 1 ? slab : 0, unroll, view_block};
    return 0;
}

void fp_clear_arm_rules() {
    std::lock_guard<std::mutex> lock(g_arm_mutex);
    g_arm_count = 0;
}

void fp_forward_arm(int D, int H, int W, int* arm, int* slab, int* unroll, int* view_block) {
    const long long voxels = (long long)D * H * W;
    std::lock_guard<std::mutex> lock(g_arm_mutex);
    for (int i = 0; i < g_arm_count; ++i)
        if (voxels <= g_arm_rules[i].voxels_max) {
            *arm = g_arm_rules[i].arm;
            *slab = g_arm_rules[i].slab;
            *unroll = g_arm_rules[i].unroll;
            *view_block = g_arm_rules[i].view_block;
            return;
        }
    // built-in choice: the L1 arm; above 2^26 voxels (512^3: 90.4 vs 94.1 ms
    // for 96 views of 768^2) CTAs in view blocks of 16, below (256^3) the
    // order makes no difference
    *arm = 0;
    *slab = 0;
    *unroll = 1;
    *view_block = voxels > (1LL << 26) ? 16 : 0;
}

FpArm fp_forward_arm(int D, int H, int W) {
    FpArm a;
    fp_forward_arm(D, H, W, &a.arm, &a.slab, &a.unroll, &a.view_block);
    return a;
}

int fp_launch_forward(const FpArgs& args, const FpTile& tile, const FpArm& a, cudaStream_t s) {
    FpArgs p = args;
    p.view_block = a.view_block;
    const bool div = !is_pow2_float(p.voxel_size);
    if (a.arm == 2 && tile.tu == 8) {
        // p.quads holds the z-pair layout (the caller built it for this arm)
        DGC_TRACE("fp_forward_pairs_kernel", s);
        const long long blocks = fp_tiles_per_view(p.U, p.V, 8) * (long long)p.A;
        const bool off = p.off_x != 0.0f || p.off_y != 0.0f || p.off_z != 0.0f;
        if (div) {
            if (off) fp_forward_pairs_kernel<8, true, true><<<(unsigned)blocks, 256, 0, s>>>(p);
            else fp_forward_pairs_kernel<8, true, false><<<(unsigned)blocks, 256, 0, s>>>(p);
        } else {
            if (off) fp_forward_pairs_kernel<8, false, true><<<(unsigned)blocks, 256, 0, s>>>(p);
            else fp_forward_pairs_kernel<8, false, false><<<(unsigned)blocks, 256, 0, s>>>(p);
        }
        DGC_LAUNCH_CHECK("fp_forward_pairs_kernel");
        return DGC_OK;
    }
    if (a.arm == 1 && tile.tu == 8) {
        bool used = false;
        const int rc = a.slab == 2 ? launch_forward_tma<2>(p, div, s, &used)
                                   : launch_forward_tma<4>(p, div, s, &used);
        if (rc != DGC_OK || used) return rc;
    }
    if (a.unroll == 2 && tile.tu == 8) return launch_forward_tu<8, 2>(p, div, s);
    switch (tile.tu) {
        case 8: return launch_forward_tu<8>(p, div, s);
        case 4: return launch_forward_tu<4>(p, div, s);
        case 2: return launch_forward_tu<2>(p, div, s);
        default:
            set_error("unsupported forward-projector tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
}

int fp_launch_backward(const FpArgs& p, const FpTile& tile, bool gradvol, cudaStream_t s) {
    switch (tile.tu) {
        case 8: return launch_backward_tu<8>(p, gradvol, s);
        case 4: return launch_backward_tu<4>(p, gradvol, s);
        case 2: return launch_backward_tu<2>(p, gradvol, s);
        default:
            set_error("unsupported backward tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
}

int fp_mse_tile(int D, int H, int W) {
    // 4 columns up to 256^3 voxels, 8 beyond: 51.0 vs 52.7 ms at 256^3 / 360 x
    // 384^2 and 5.84 vs 6.06 ms at 128^3 / 180 x 256^2, but 1145 vs 930 ms at
    // 512^3 / 720 x 768^2
    return (long long)D * H * W <= 256LL * 256 * 256 ? 4 : 8;
}

namespace {
template <int TU>
int launch_mse_grad_tu(const FpArgs& p, const float* measured, const float* mask, float scale,
                       double* loss_partials, cudaStream_t s) {
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    const bool div = !is_pow2_float(p.voxel_size);
    const bool off = p.off_x != 0.0f || p.off_y != 0.0f || p.off_z != 0.0f;
    if (div) {
        if (off) fp_mse_grad_kernel<TU, true, true><<<(unsigned)blocks, 256, 0, s>>>(p, measured, mask, scale, loss_partials);
        else fp_mse_grad_kernel<TU, true, false><<<(unsigned)blocks, 256, 0, s>>>(p, measured, mask, scale, loss_partials);
    } else {
        if (off) fp_mse_grad_kernel<TU, false, true><<<(unsigned)blocks, 256, 0, s>>>(p, measured, mask, scale, loss_partials);
        else fp_mse_grad_kernel<TU, false, false><<<(unsigned)blocks, 256, 0, s>>>(p, measured, mask, scale, loss_partials);
    }
    DGC_LAUNCH_CHECK("fp_mse_grad_kernel");
    return DGC_OK;
}
}  // namespace

int fp_launch_mse_grad(const FpArgs& p, int tile, const float* measured, const float* mask,
                       float scale, double* loss_partials, cudaStream_t s) {
    DGC_TRACE("fp_mse_grad_kernel", s);
    switch (tile) {
        case 4: return launch_mse_grad_tu<4>(p, measured, mask, scale, loss_partials, s);
        case 2: return launch_mse_grad_tu<2>(p, measured, mask, scale, loss_partials, s);
        default: return launch_mse_grad_tu<8>(p, measured, mask, scale, loss_partials, s);
    }
}

int fp_sum_partials(const double* x, long long n, double scale, double* out, cudaStream_t s) {
    DGC_TRACE("sum_partials", s);
    sum_partials_kernel<<<1, 256, 0, s>>>(x, n, scale, out);
    DGC_LAUNCH_CHECK("sum_partials");
    return DGC_OK;
}

int fp_launch_counts(const FpArgs& p, int64_t* counts, cudaStream_t s) {
    DGC_TRACE("fp_count_kernel", s);
    const long long blocks = (long long)p.A * ceil_div(p.U, 8) * ceil_div(p.V, 32);
    fp_count_kernel<<<(unsigned)blocks, 256, 0, s>>>(p, counts);
    DGC_LAUNCH_CHECK("fp_count_kernel");
    return DGC_OK;
}

int fp_reduce_partials(const double* partials, int A, long long tiles, const GeometryGrad& out,
                       cudaStream_t s) {
    DGC_TRACE("reduce_view_partials", s);
    reduce_view_partials_kernel<<<A, 256, 0, s>>>(partials, (int)tiles, out);
    DGC_LAUNCH_CHECK("reduce_view_partials");
    return DGC_OK;
}

// ------------------------------------------------------------ batched launches

int batch_launch_quads(const BatchTables& t, long long blocks, cudaStream_t s) {
    DGC_TRACE("batch_quads", s);
    batch_quads_kernel<<<(unsigned)blocks, dim3(32, 8), 0, s>>>(t);
    DGC_LAUNCH_CHECK("batch_quads");
    return DGC_OK;
}

int batch_launch_forward(const BatchTables& t, int grid, cudaStream_t s) {
    DGC_TRACE("batch_forward_kernel", s);
    DGC_CUDA(cudaMemsetAsync(t.counters, 0, sizeof(unsigned long long), s));
    batch_forward_kernel<<<grid, 256, 0, s>>>(t);
    DGC_LAUNCH_CHECK("batch_forward_kernel");
    return DGC_OK;
}

int batch_launch_backward(const BatchTables& t, int grid, long long views, long long fold_blocks,
                          cudaStream_t s) {
    {
        DGC_TRACE("batch_backward_kernel", s);
        DGC_CUDA(cudaMemsetAsync(t.counters + 1, 0, sizeof(unsigned long long), s));
        batch_backward_kernel<<<grid, 256, 0, s>>>(t);
        DGC_LAUNCH_CHECK("batch_backward_kernel");
    }
    {
        DGC_TRACE("batch_reduce", s);
        batch_reduce_kernel<<<(unsigned)views, 256, 0, s>>>(t);
        DGC_LAUNCH_CHECK("batch_reduce");
    }
    if (fold_blocks > 0) {
        DGC_TRACE("batch_fold", s);
        batch_fold_kernel<<<(unsigned)fold_blocks, 256, 0, s>>>(t);
        DGC_LAUNCH_CHECK("batch_fold");
    }
    return DGC_OK;
}

int batch_persistent_grid(bool backward, int* grid) {
    int dev = 0, sms = 0, per_sm = 0;
    DGC_CUDA(cudaGetDevice(&dev));
    DGC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (backward)
        DGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_backward_kernel, 256, 0));
    else
        DGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_forward_kernel, 256, 0));
    *grid = std::max(1, per_sm) * sms;
    return DGC_OK;
}

}  // namespace dgc
