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
#include "common.cuh"
#include "forward_projector.cuh"

namespace dgc {

// ---------------------------------------------------------------------------
// Volume re-layout: [D][H][W] -> Z-fastest edge-replicated quads
// ---------------------------------------------------------------------------

// grid: x = ceil((W+1)/32) * (H+1), y = ceil((D+2)/32); block (32, 8)
__global__ void build_volume_quads_kernel(const float* __restrict__ vol, int D, int H, int W,
                                          float4* __restrict__ Q) {
    __shared__ float4 tile[32][33];
    const int xtiles = (W + 1 + 31) / 32;
    const int yp = blockIdx.x / xtiles;
    const int xp0 = (blockIdx.x - yp * xtiles) * 32;
    const int zp0 = blockIdx.y * 32;
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

int build_volume_quads(const float* vol, int D, int H, int W, float4* quads, cudaStream_t s) {
    DGC_TRACE("build_volume_quads", s);
    const dim3 grid((unsigned)(ceil_div(W + 1, 32) * (long long)(H + 1)), (unsigned)ceil_div(D + 2, 32));
    build_volume_quads_kernel<<<grid, dim3(32, 8), 0, s>>>(vol, D, H, W, quads);
    DGC_LAUNCH_CHECK("build_volume_quads");
    return DGC_OK;
}

// ---------------------------------------------------------------------------
// Per-view and per-ray set-up (reference arithmetic, kept expression for
// expression so that t_min / t_max -- and with them the FP32 sample count --
// agree with the reference kernel)
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
    vg.ox = -vg.sod * vg.s + g.src_x[a];
    vg.oy = vg.sod * vg.c + g.src_y[a];
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
    const float tx = u_phys * vg.c - vg.dn * vg.s;
    const float ty = u_phys * vg.s + vg.dn * vg.c;
    const float tz = v_phys;
    const float rx = tx - vg.ox, ry = ty - vg.oy, rz = tz - vg.oz;
    r.len = sqrtf(rx * rx + ry * ry + rz * rz);
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
    const float bxl = (-p.W * 0.5f - 0.5f) * p.voxel_size + p.off_x;
    const float byl = (-p.H * 0.5f - 0.5f) * p.voxel_size + p.off_y;
    const float bzl = (-p.D * 0.5f - 0.5f) * p.voxel_size + p.off_z;
    const float bxh = (p.W * 0.5f - 0.5f) * p.voxel_size + p.off_x;
    const float byh = (p.H * 0.5f - 0.5f) * p.voxel_size + p.off_y;
    const float bzh = (p.D * 0.5f - 0.5f) * p.voxel_size + p.off_z;
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
    const float x0 = to_voxel<DIV>(vg.ox + r.tmin * r.dx, p.off_x, p.voxel_size, p.inv_voxel, hx);
    const float x1 = to_voxel<DIV>(vg.ox + r.tmax * r.dx, p.off_x, p.voxel_size, p.inv_voxel, hx);
    const float y0 = to_voxel<DIV>(vg.oy + r.tmin * r.dy, p.off_y, p.voxel_size, p.inv_voxel, hy);
    const float y1 = to_voxel<DIV>(vg.oy + r.tmax * r.dy, p.off_y, p.voxel_size, p.inv_voxel, hy);
    const float z0 = to_voxel<DIV>(vg.oz + r.tmin * r.dz, p.off_z, p.voxel_size, p.inv_voxel, hz);
    const float z1 = to_voxel<DIV>(vg.oz + r.tmax * r.dz, p.off_z, p.voxel_size, p.inv_voxel, hz);
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

__device__ __forceinline__ uint32_t quad_index(const Cell& c, const FpArgs& p) {
    return c.bz + c.bx * p.zq_x + c.by * p.zq_y + p.zq_bias;
}

// Sum of the trilinear samples along the ray (fp.cu:321-335).  The quads
// hold the y-pairs of x0 and x1 as 64-bit halves, so the interpolation runs
// as packed pairs: along x for (y0, y1) at z0 and z1, along z, then along y.
template <bool CLAMP, bool DIV, bool OFF>
__device__ __forceinline__ float march_sum(const RaySetup& r, const ViewGeo& vg, const FpArgs& p) {
    const float hx = p.W * 0.5f, hy = p.H * 0.5f, hz = p.D * 0.5f;
    const ulonglong2* __restrict__ Q = reinterpret_cast<const ulonglong2*>(p.quads);
    const int nmax = step_bound(r, p.step_size);
    float acc = 0.0f;
    float t = r.tmin;
    int n = 0;
#pragma unroll 1
    for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
        const float px = vg.ox + t * r.dx;
        const float py = vg.oy + t * r.dy;
        const float pz = vg.oz + t * r.dz;
        const Cell c =
            locate<CLAMP>(to_voxel<DIV, OFF>(px, p.off_x, p.voxel_size, p.inv_voxel, hx),
                          to_voxel<DIV, OFF>(py, p.off_y, p.voxel_size, p.inv_voxel, hy),
                          to_voxel<DIV, OFF>(pz, p.off_z, p.voxel_size, p.inv_voxel, hz), p);
        const uint32_t qi = quad_index(c, p);
        const ulonglong2 q0 = __ldg(Q + qi);
        const ulonglong2 q1 = __ldg(Q + qi + 1);
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

__device__ __forceinline__ TileCoord tile_coord(const FpArgs& p, int tiles_u) {
    int b = blockIdx.x;
    TileCoord tc;
    tc.tu = b % tiles_u;
    b /= tiles_u;
    tc.a = b % p.A;
    tc.tv = b / p.A;
    return tc;
}

// ---------------------------------------------------------------------------
// Forward kernel
// ---------------------------------------------------------------------------

// A CTA owns TU detector columns x (256/TU) rows of one view; warps run along
// V (32 consecutive rows of one column).
template <int TU, bool DIV, bool OFF>
__global__ void __launch_bounds__(256) fp_forward_kernel(FpArgs p) {
    constexpr int TV = 256 / TU;
    constexpr int WARPS_V = TV / 32;
    static_assert(TV % 32 == 0, "rows per CTA must be whole warps");
    __shared__ ViewGeo s_view;
    const int tiles_u = (p.U + TU - 1) / TU;
    const TileCoord tc = tile_coord(p, tiles_u);
    if (threadIdx.x == 0) load_view(p.g, tc.a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = tc.tu * TU + warp / WARPS_V;
    const int v = tc.tv * TV + (warp % WARPS_V) * 32 + lane;
    if (u >= p.U || v >= p.V) return;

    const RaySetup r = setup_ray(vg, u, v, p);
    float integral = 0.0f;
    if (r.ok && r.hit) {
        integral = ray_inside_pad<DIV>(r, vg, p) ? march_sum<false, DIV, OFF>(r, vg, p)
                                                 : march_sum<true, DIV, OFF>(r, vg, p);
        integral *= p.step_size;
    }
    p.projections[((long long)tc.a * p.U + u) * p.V + v] = integral;
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

template <bool CLAMP, bool GRADVOL>
__device__ __forceinline__ RayGrad march_grad(const RaySetup& r, const ViewGeo& vg,
                                              const FpArgs& p, float gs) {
    const float hx = p.W * 0.5f, hy = p.H * 0.5f, hz = p.D * 0.5f;
    const float4* __restrict__ Q = p.quads;
    RayGrad rg{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int nmax = step_bound(r, p.step_size);
    float t = r.tmin;
    int n = 0;
#pragma unroll 1
    for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
        const float px = vg.ox + t * r.dx;
        const float py = vg.oy + t * r.dy;
        const float pz = vg.oz + t * r.dz;
        const Cell c = locate<CLAMP>(to_voxel<false>(px, p.off_x, p.voxel_size, p.inv_voxel, hx),
                                     to_voxel<false>(py, p.off_y, p.voxel_size, p.inv_voxel, hy),
                                     to_voxel<false>(pz, p.off_z, p.voxel_size, p.inv_voxel, hz), p);
        const uint32_t qi = quad_index(c, p);
        const float4 q0 = __ldg(Q + qi);
        const float4 q1 = __ldg(Q + qi + 1);
        // d/dx, d/dy, d/dz of the trilinear interpolant (voxel units); quad
        // components are (x0y0, x0y1, x1y0, x1y1)
        const float gx = lerpf(lerpf(q0.z - q0.x, q0.w - q0.y, c.fy),
                               lerpf(q1.z - q1.x, q1.w - q1.y, c.fy), c.fz);
        const float gy = lerpf(lerpf(q0.y - q0.x, q0.w - q0.z, c.fx),
                               lerpf(q1.y - q1.x, q1.w - q1.z, c.fx), c.fz);
        const float gz = lerpf(lerpf(q1.x - q0.x, q1.z - q0.z, c.fx),
                               lerpf(q1.y - q0.y, q1.w - q0.w, c.fx), c.fy);
        const float tau = t - r.tmin;
        rg.s1x += gx;
        rg.s1y += gy;
        rg.s1z += gz;
        rg.s2x = fmaf(gx, tau, rg.s2x);
        rg.s2y = fmaf(gy, tau, rg.s2y);
        rg.s2z = fmaf(gz, tau, rg.s2z);
        if (GRADVOL) {
            // adjoint of the trilinear sample (fp.cu:231-240), padded z-fastest buffer
            const float mx = 1.0f - c.fx, my = 1.0f - c.fy, mz = 1.0f - c.fz;
            const float gy0 = gs * my, gy1 = gs * c.fy;
            const float w00 = gy0 * mx, w01 = gy0 * c.fx, w10 = gy1 * mx, w11 = gy1 * c.fx;
            float* g0 = p.grad_pad + (c.bz + c.bx * p.gz_x + c.by * p.gz_y + p.gz_bias);
            float* g1 = g0 + p.gz_y;
            atomicAdd(g0, w00 * mz);
            atomicAdd(g0 + 1, w00 * c.fz);
            atomicAdd(g0 + p.gz_x, w01 * mz);
            atomicAdd(g0 + p.gz_x + 1, w01 * c.fz);
            atomicAdd(g1, w10 * mz);
            atomicAdd(g1 + 1, w10 * c.fz);
            atomicAdd(g1 + p.gz_x, w11 * mz);
            atomicAdd(g1 + p.gz_x + 1, w11 * c.fz);
        }
    }
    return rg;
}

template <int TU, bool GRADVOL>
__global__ void __launch_bounds__(256) fp_backward_kernel(FpArgs p) {
    constexpr int TV = 256 / TU;
    constexpr int WARPS_V = TV / 32;
    static_assert(TV % 32 == 0, "rows per CTA must be whole warps");
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
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = tc.tu * TU + warp / WARPS_V;
    const int v = tc.tv * TV + (warp % WARPS_V) * 32 + lane;

    float terms[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const bool in_range = u < p.U && v < p.V;
    const float grad_out =
        in_range ? p.grad_projections[((long long)a * p.U + u) * p.V + v] : 0.0f;
    // fp.cu:381 -- rays with a zero upstream gradient contribute nothing.
    if (in_range && grad_out != 0.0f) {
        const RaySetup r = setup_ray(vg, u, v, p);
        if (r.ok) {
            // Gradients wrt the ray origin (direct part) and the target point.
            float godx = 0.f, gody = 0.f, godz = 0.f;
            float grx = 0.f, gry = 0.f, grz = 0.f;
            if (r.hit) {
                const float gs = grad_out * p.step_size;
                const RayGrad rg = ray_inside_pad<false>(r, vg, p)
                                       ? march_grad<false, GRADVOL>(r, vg, p, gs)
                                       : march_grad<true, GRADVOL>(r, vg, p, gs);
                // fp.cu:441-467 give, with G = gs/voxel,
                //   grad_origin_direct = G*s1 - (G*(s1.d)/d_e) e_e
                //   grad_direction     = G*sum g*t - (G*(s1.d) t_min/d_e) e_e
                // (e = entry axis).  Writing sum g*t = s2 + t_min*s1 and
                //   q = s1 - ((s1.d)/d_e) e_e   (so q.d = 0)
                // gives grad_origin_direct = G*q and grad_direction = G*(s2 + t_min*q):
                // the same values without the large t_min*s1 terms that cancel.
                float qx = rg.s1x, qy = rg.s1y, qz = rg.s1z;
                if (r.entry_axis == 0) qx = -(rg.s1y * r.dy + rg.s1z * r.dz) / r.dx;
                else if (r.entry_axis == 1) qy = -(rg.s1x * r.dx + rg.s1z * r.dz) / r.dy;
                else if (r.entry_axis == 2) qz = -(rg.s1x * r.dx + rg.s1y * r.dy) / r.dz;
                const float G = gs * p.inv_voxel;
                godx = G * qx;
                gody = G * qy;
                godz = G * qz;
                // fp.cu:470-486: chain through direction = normalize(target - origin);
                // q is orthogonal to d, so only s2 loses its component along d.
                const float ds2 = r.dx * rg.s2x + r.dy * rg.s2y + r.dz * rg.s2z;
                const float k = G / r.len;
                grx = k * (rg.s2x - r.dx * ds2 + r.tmin * qx);
                gry = k * (rg.s2y - r.dy * ds2 + r.tmin * qy);
                grz = k * (rg.s2z - r.dz * ds2 + r.tmin * qz);
            }
            const float gox = godx - grx, goy = gody - gry, goz = godz - grz;
            // fp.cu:488-527: per-view geometry terms.
            const float u_phys = (u - vg.u0) * p.pixel_size;
            const float dOx = -vg.sod * vg.c, dOy = -vg.sod * vg.s;
            const float dTx = -u_phys * vg.s - vg.dn * vg.c;
            const float dTy = u_phys * vg.c - vg.dn * vg.s;
            terms[0] = gox * dOx + goy * dOy + grx * dTx + gry * dTy;
            terms[1] = grx * vg.s - gry * vg.c;
            terms[2] = (gox + grx) * (-vg.s) + (goy + gry) * vg.c;
            terms[3] = -p.pixel_size * (grx * vg.c + gry * vg.s);
            terms[4] = -p.pixel_size * grz;
            terms[5] = gox;
            terms[6] = goy;
            terms[7] = goz;
        }
    }
    // Fixed-order FP64 reduction of the eight terms over the CTA.
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
        p.partials[((long long)a * tiles + tile) * 8 + threadIdx.x] = acc;
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

// grad_volume[z,y,x] = sum of the padded cells that clamp onto (z,y,x); the
// padded buffer is z-fastest: G[(yp*(W+2) + xp)*(D+2) + zp].
__global__ void fold_padded_gradient_kernel(const float* __restrict__ gpad, int D, int H, int W,
                                            float* __restrict__ grad) {
    const long long PZ = D + 2, PX = W + 2;
    const long long total = (long long)D * H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
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
                    acc += gpad[((long long)ys[iy] * PX + xs[ix]) * PZ + zs[iz]];
        grad[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// Launch configuration
// ---------------------------------------------------------------------------

namespace {

template <int TU>
int launch_forward_tu(const FpArgs& p, bool div, cudaStream_t s) {
    DGC_TRACE("fp_forward_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    const bool off = p.off_x != 0.0f || p.off_y != 0.0f || p.off_z != 0.0f;
    if (div) {
        if (off) fp_forward_kernel<TU, true, true><<<(unsigned)blocks, 256, 0, s>>>(p);
        else fp_forward_kernel<TU, true, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    } else {
        if (off) fp_forward_kernel<TU, false, true><<<(unsigned)blocks, 256, 0, s>>>(p);
        else fp_forward_kernel<TU, false, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    }
    DGC_LAUNCH_CHECK("fp_forward_kernel");
    return DGC_OK;
}

template <int TU>
int launch_backward_tu(const FpArgs& p, bool gradvol, cudaStream_t s) {
    DGC_TRACE(gradvol ? "fp_backward_kernel<gradvol>" : "fp_backward_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    if (gradvol)
        fp_backward_kernel<TU, true><<<(unsigned)blocks, 256, 0, s>>>(p);
    else
        fp_backward_kernel<TU, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fp_backward_kernel");
    return DGC_OK;
}

}  // namespace

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
    // padded gradient: G[(yp*(W+2) + xp)*(D+2) + zp]
    p.gz_x = (uint32_t)(p.D + 2);
    p.gz_y = (uint32_t)(p.W + 2) * (uint32_t)(p.D + 2);
    p.gz_bias = (1u + p.gz_x + p.gz_y) - kFloorMagicBits * (1u + p.gz_x + p.gz_y);
    p.inv_voxel = 1.0f / p.voxel_size;
}

int fp_launch_forward(const FpArgs& p, const FpTile& tile, cudaStream_t s) {
    const bool div = !is_pow2_float(p.voxel_size);
    switch (tile.tu) {
        case 8: return launch_forward_tu<8>(p, div, s);
        case 4: return launch_forward_tu<4>(p, div, s);
        default:
            set_error("unsupported forward-projector tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
}

int fp_launch_backward(const FpArgs& p, const FpTile& tile, bool gradvol, cudaStream_t s) {
    switch (tile.tu) {
        case 8: return launch_backward_tu<8>(p, gradvol, s);
        case 4: return launch_backward_tu<4>(p, gradvol, s);
        default:
            set_error("unsupported backward tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
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

int fp_fold_gradient(const float* gpad, int D, int H, int W, float* grad, cudaStream_t s) {
    DGC_TRACE("fold_padded_gradient", s);
    const long long total = (long long)D * H * W;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    fold_padded_gradient_kernel<<<blocks, 256, 0, s>>>(gpad, D, H, W, grad);
    DGC_LAUNCH_CHECK("fold_padded_gradient");
    return DGC_OK;
}

}  // namespace dgc
