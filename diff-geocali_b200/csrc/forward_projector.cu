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
//   * The volume is re-laid out once per call into an edge-replicated,
//     quad-packed copy Q[z+1][y+1][x+1] = float4(v(z,y,x), v(z,y,x+1),
//     v(z,y+1,x), v(z,y+1,x+1)) (indices clamped), so one trilinear sample is
//     two 16-byte loads and needs no per-corner clamping: clamping the sample
//     coordinate to [-1, n-1] reproduces the reference's clamped-neighbour
//     values exactly (both neighbours of an out-of-range coordinate hold the
//     same edge value).
//   * floor() runs on the FP32 add pipe (round-down add of 1.5*2^23).
//   * A CTA owns one view and a TU x TV tile of rays; the view's source
//     position and trig live in shared memory.
//   * Geometry gradients are reduced per CTA in FP64 with warp shuffles and a
//     fixed-order tree, then per view over CTAs in a second fixed-order pass:
//     the eight per-view gradients are bitwise reproducible.
//   * The volume gradient is scattered into an edge-padded buffer and folded
//     back onto the clamped edge voxels afterwards (same sums as the
//     reference's clamped-index atomics).
#include "common.cuh"
#include "forward_projector.cuh"

namespace dgc {

// ---------------------------------------------------------------------------
// Volume re-layout
// ---------------------------------------------------------------------------

__global__ void build_volume_quads_kernel(const float* __restrict__ vol, int D, int H, int W,
                                          float4* __restrict__ quads) {
    const int QW = W + 1, QH = H + 1;
    const long long total = (long long)(D + 2) * QH * QW;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int xp = (int)(i % QW);
        const long long r = i / QW;
        const int yp = (int)(r % QH);
        const int zp = (int)(r / QH);
        const int z = min(max(zp - 1, 0), D - 1);
        const int y0 = min(max(yp - 1, 0), H - 1), y1 = min(yp, H - 1);
        const int x0 = min(max(xp - 1, 0), W - 1), x1 = min(xp, W - 1);
        const float* plane = vol + (long long)z * H * W;
        float4 q;
        q.x = __ldg(plane + (long long)y0 * W + x0);
        q.y = __ldg(plane + (long long)y0 * W + x1);
        q.z = __ldg(plane + (long long)y1 * W + x0);
        q.w = __ldg(plane + (long long)y1 * W + x1);
        quads[i] = q;
    }
}

int build_volume_quads(const float* vol, int D, int H, int W, float4* quads, cudaStream_t s) {
    DGC_TRACE("build_volume_quads", s);
    const long long total = (long long)(D + 2) * (H + 1) * (W + 1);
    const int threads = 256;
    const int blocks = (int)std::min<long long>((total + threads - 1) / threads, 148LL * 16);
    build_volume_quads_kernel<<<blocks, threads, 0, s>>>(vol, D, H, W, quads);
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
template <bool DIV>
__device__ __forceinline__ float to_voxel(float pos, float off, float voxel, float inv_voxel,
                                          float half) {
    if (DIV) return __fdiv_rn(pos - off, voxel) + half;
    return fmaf(pos - off, inv_voxel, half);
}

struct Corner {
    uint32_t qi;  // quad index of the (z0, y0, x0) cell in the padded layout
    float fx, fy, fz;
    uint32_t bx, by, bz;  // biased floors (for the padded scalar index)
};

__device__ __forceinline__ Corner locate(float x, float y, float z, const FpArgs& p) {
    // Clamp to [-1, n-1]: beyond that both neighbours are edge replicas.
    x = fminf(fmaxf(x, -1.0f), (float)(p.W - 1));
    y = fminf(fmaxf(y, -1.0f), (float)(p.H - 1));
    z = fminf(fmaxf(z, -1.0f), (float)(p.D - 1));
    const FloorSplit sx = floor_split(x), sy = floor_split(y), sz = floor_split(z);
    Corner c;
    c.fx = sx.frac;
    c.fy = sy.frac;
    c.fz = sz.frac;
    c.bx = sx.biased;
    c.by = sy.biased;
    c.bz = sz.biased;
    c.qi = sz.biased * p.q_plane + sy.biased * p.q_row + sx.biased + p.q_bias;
    return c;
}

// ---------------------------------------------------------------------------
// Forward kernel
// ---------------------------------------------------------------------------

template <int TU, int WU, bool DIV>
__global__ void __launch_bounds__(256) fp_forward_kernel(FpArgs p) {
    constexpr int TV = 256 / TU;
    constexpr int WV = 32 / WU;
    constexpr int WARPS_V = TV / WV;
    __shared__ ViewGeo s_view;
    const int tiles_v = (p.V + TV - 1) / TV;
    const int tiles = ((p.U + TU - 1) / TU) * tiles_v;
    const int a = blockIdx.x / tiles;
    const int tile = blockIdx.x - a * tiles;
    if (threadIdx.x == 0) load_view(p.g, a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = (tile / tiles_v) * TU + (warp / WARPS_V) * WU + lane / WV;
    const int v = (tile % tiles_v) * TV + (warp % WARPS_V) * WV + lane % WV;
    if (u >= p.U || v >= p.V) return;

    const RaySetup r = setup_ray(vg, u, v, p);
    float integral = 0.0f;
    if (r.ok && r.hit) {
        const float hx = p.W * 0.5f, hy = p.H * 0.5f, hz = p.D * 0.5f;
        const float4* __restrict__ Q = p.quads;
        const int nmax = step_bound(r, p.step_size);
        float t = r.tmin;
        int n = 0;
#pragma unroll 1
        for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
            const float px = vg.ox + t * r.dx;
            const float py = vg.oy + t * r.dy;
            const float pz = vg.oz + t * r.dz;
            const float x = to_voxel<DIV>(px, p.off_x, p.voxel_size, p.inv_voxel, hx);
            const float y = to_voxel<DIV>(py, p.off_y, p.voxel_size, p.inv_voxel, hy);
            const float z = to_voxel<DIV>(pz, p.off_z, p.voxel_size, p.inv_voxel, hz);
            const Corner c = locate(x, y, z, p);
            const float4 q0 = __ldg(Q + c.qi);
            const float4 q1 = __ldg(Q + c.qi + p.q_plane);
            const float c0 = lerpf(lerpf(q0.x, q0.y, c.fx), lerpf(q0.z, q0.w, c.fx), c.fy);
            const float c1 = lerpf(lerpf(q1.x, q1.y, c.fx), lerpf(q1.z, q1.w, c.fx), c.fy);
            integral += lerpf(c0, c1, c.fz);
        }
        integral *= p.step_size;
    }
    p.projections[((long long)a * p.U + u) * p.V + v] = integral;
}

// Sample counts under the same FP32 rule (measurement support).
__global__ void __launch_bounds__(256) fp_count_kernel(FpArgs p, int64_t* __restrict__ counts) {
    constexpr int TU = 16, TV = 16;
    __shared__ ViewGeo s_view;
    const int tiles_v = (p.V + TV - 1) / TV;
    const int tiles = ((p.U + TU - 1) / TU) * tiles_v;
    const int a = blockIdx.x / tiles;
    const int tile = blockIdx.x - a * tiles;
    if (threadIdx.x == 0) load_view(p.g, a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    const int u = (tile / tiles_v) * TU + threadIdx.x / TV;
    const int v = (tile % tiles_v) * TV + threadIdx.x % TV;
    if (u >= p.U || v >= p.V) return;
    const RaySetup r = setup_ray(vg, u, v, p);
    long long n = 0;
    if (r.ok && r.hit) {
        const int nmax = step_bound(r, p.step_size);
        for (float t = r.tmin; t <= r.tmax && n < nmax; t += p.step_size) ++n;
    }
    counts[((long long)a * p.U + u) * p.V + v] = n;
}

// ---------------------------------------------------------------------------
// Backward kernel: volume adjoint (optional) + per-ray geometry terms
// ---------------------------------------------------------------------------

template <int TU, int WU, bool GRADVOL>
__global__ void __launch_bounds__(256) fp_backward_kernel(FpArgs p) {
    constexpr int TV = 256 / TU;
    constexpr int WV = 32 / WU;
    constexpr int WARPS_V = TV / WV;
    __shared__ ViewGeo s_view;
    __shared__ double s_red[8][8];
    const int tiles_v = (p.V + TV - 1) / TV;
    const int tiles = ((p.U + TU - 1) / TU) * tiles_v;
    const int a = blockIdx.x / tiles;
    const int tile = blockIdx.x - a * tiles;
    if (threadIdx.x == 0) load_view(p.g, a, s_view);
    __syncthreads();
    const ViewGeo vg = s_view;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int u = (tile / tiles_v) * TU + (warp / WARPS_V) * WU + lane / WV;
    const int v = (tile % tiles_v) * TV + (warp % WARPS_V) * WV + lane % WV;

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
                const float hx = p.W * 0.5f, hy = p.H * 0.5f, hz = p.D * 0.5f;
                const float4* __restrict__ Q = p.quads;
                // s1 = sum of the voxel-unit spatial gradient g over the samples,
                // s2 = sum of g * (t - t_min).
                float s1x = 0.f, s1y = 0.f, s1z = 0.f, s2x = 0.f, s2y = 0.f, s2z = 0.f;
                const int nmax = step_bound(r, p.step_size);
                float t = r.tmin;
                int n = 0;
#pragma unroll 1
                for (; t <= r.tmax && n < nmax; t += p.step_size, ++n) {
                    const float px = vg.ox + t * r.dx;
                    const float py = vg.oy + t * r.dy;
                    const float pz = vg.oz + t * r.dz;
                    const float x = to_voxel<false>(px, p.off_x, p.voxel_size, p.inv_voxel, hx);
                    const float y = to_voxel<false>(py, p.off_y, p.voxel_size, p.inv_voxel, hy);
                    const float z = to_voxel<false>(pz, p.off_z, p.voxel_size, p.inv_voxel, hz);
                    const Corner c = locate(x, y, z, p);
                    const float4 q0 = __ldg(Q + c.qi);
                    const float4 q1 = __ldg(Q + c.qi + p.q_plane);
                    // d/dx, d/dy, d/dz of the trilinear interpolant (voxel units)
                    const float gx = lerpf(lerpf(q0.y - q0.x, q0.w - q0.z, c.fy),
                                           lerpf(q1.y - q1.x, q1.w - q1.z, c.fy), c.fz);
                    const float gy = lerpf(lerpf(q0.z - q0.x, q0.w - q0.y, c.fx),
                                           lerpf(q1.z - q1.x, q1.w - q1.y, c.fx), c.fz);
                    const float gz = lerpf(lerpf(q1.x - q0.x, q1.y - q0.y, c.fx),
                                           lerpf(q1.z - q0.z, q1.w - q0.w, c.fx), c.fy);
                    const float tau = t - r.tmin;
                    s1x += gx;
                    s1y += gy;
                    s1z += gz;
                    s2x = fmaf(gx, tau, s2x);
                    s2y = fmaf(gy, tau, s2y);
                    s2z = fmaf(gz, tau, s2z);
                    if (GRADVOL) {
                        const float mx = 1.0f - c.fx, my = 1.0f - c.fy, mz = 1.0f - c.fz;
                        const float g0 = gs * mz, g1 = gs * c.fz;
                        const float g00 = g0 * my, g10 = g0 * c.fy, g01 = g1 * my, g11 = g1 * c.fy;
                        float* gp = p.grad_pad + (c.bz * p.g_plane + c.by * p.g_row + c.bx + p.g_bias);
                        atomicAdd(gp, g00 * mx);
                        atomicAdd(gp + 1, g00 * c.fx);
                        atomicAdd(gp + p.g_row, g10 * mx);
                        atomicAdd(gp + p.g_row + 1, g10 * c.fx);
                        atomicAdd(gp + p.g_plane, g01 * mx);
                        atomicAdd(gp + p.g_plane + 1, g01 * c.fx);
                        atomicAdd(gp + p.g_plane + p.g_row, g11 * mx);
                        atomicAdd(gp + p.g_plane + p.g_row + 1, g11 * c.fx);
                    }
                }
                // fp.cu:441-467 give, with G = gs/voxel,
                //   grad_origin_direct = G*s1 - (G*(s1.d)/d_e) e_e
                //   grad_direction     = G*sum g*t - (G*(s1.d) t_min/d_e) e_e
                // (e = entry axis).  Writing sum g*t = s2 + t_min*s1 and
                //   q = s1 - ((s1.d)/d_e) e_e   (so q.d = 0)
                // gives grad_origin_direct = G*q and grad_direction = G*(s2 + t_min*q):
                // the same values without the large t_min*s1 terms that cancel.
                float qx = s1x, qy = s1y, qz = s1z;
                if (r.entry_axis == 0) qx = -(s1y * r.dy + s1z * r.dz) / r.dx;
                else if (r.entry_axis == 1) qy = -(s1x * r.dx + s1z * r.dz) / r.dy;
                else if (r.entry_axis == 2) qz = -(s1x * r.dx + s1y * r.dy) / r.dz;
                const float G = gs * p.inv_voxel;
                godx = G * qx;
                gody = G * qy;
                godz = G * qz;
                // fp.cu:470-486: chain through direction = normalize(target - origin);
                // q is orthogonal to d, so only s2 loses its component along d.
                const float ds2 = r.dx * s2x + r.dy * s2y + r.dz * s2z;
                const float k = G / r.len;
                grx = k * (s2x - r.dx * ds2 + r.tmin * qx);
                gry = k * (s2y - r.dy * ds2 + r.tmin * qy);
                grz = k * (s2z - r.dz * ds2 + r.tmin * qz);
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

// grad_volume[z,y,x] = sum of the padded cells that clamp onto (z,y,x).
__global__ void fold_padded_gradient_kernel(const float* __restrict__ gpad, int D, int H, int W,
                                            float* __restrict__ grad) {
    const int PW = W + 2, PH = H + 2;
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
        for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
                for (int ix = 0; ix < nx; ++ix)
                    acc += gpad[((long long)zs[iz] * PH + ys[iy]) * PW + xs[ix]];
        grad[i] = acc;
    }
}

// ---------------------------------------------------------------------------
// Launch configuration
// ---------------------------------------------------------------------------

namespace {

template <int TU, int WU>
int launch_forward_tu(const FpArgs& p, bool div, cudaStream_t s) {
    DGC_TRACE("fp_forward_kernel", s);
    constexpr int TV = 256 / TU;
    const long long blocks = (long long)p.A * ceil_div(p.U, TU) * ceil_div(p.V, TV);
    if (div)
        fp_forward_kernel<TU, WU, true><<<(unsigned)blocks, 256, 0, s>>>(p);
    else
        fp_forward_kernel<TU, WU, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fp_forward_kernel");
    return DGC_OK;
}

template <int TU, int WU>
int launch_backward_tu(const FpArgs& p, bool gradvol, cudaStream_t s) {
    DGC_TRACE(gradvol ? "fp_backward_kernel<gradvol>" : "fp_backward_kernel", s);
    const long long blocks = fp_tiles_per_view(p.U, p.V, TU) * (long long)p.A;
    if (gradvol)
        fp_backward_kernel<TU, WU, true><<<(unsigned)blocks, 256, 0, s>>>(p);
    else
        fp_backward_kernel<TU, WU, false><<<(unsigned)blocks, 256, 0, s>>>(p);
    DGC_LAUNCH_CHECK("fp_backward_kernel");
    return DGC_OK;
}

}  // namespace

long long fp_tiles_per_view(int U, int V, int tu) {
    const int tv = 256 / tu;
    return (long long)ceil_div(U, tu) * ceil_div(V, tv);
}

void fp_fill_layout(FpArgs& p) {
    p.q_row = (uint32_t)(p.W + 1);
    p.q_plane = (uint32_t)(p.H + 1) * (uint32_t)(p.W + 1);
    // quad index of (z0+1, y0+1, x0+1) from the biased floors
    p.q_bias = (uint32_t)(1u + p.q_row + p.q_plane) -
               kFloorMagicBits * (p.q_plane + p.q_row + 1u);
    p.g_row = (uint32_t)(p.W + 2);
    p.g_plane = (uint32_t)(p.H + 2) * (uint32_t)(p.W + 2);
    p.g_bias = (uint32_t)(1u + p.g_row + p.g_plane) -
               kFloorMagicBits * (p.g_plane + p.g_row + 1u);
    p.inv_voxel = 1.0f / p.voxel_size;
}

int fp_launch_forward(const FpArgs& p, const FpTile& tile, cudaStream_t s) {
    const bool div = !is_pow2_float(p.voxel_size);
    switch (tile.tu * 100 + tile.wu) {
        case 1608: return launch_forward_tu<16, 8>(p, div, s);
        case 1604: return launch_forward_tu<16, 4>(p, div, s);
        case 1616: return launch_forward_tu<16, 16>(p, div, s);
        case 3232: return launch_forward_tu<32, 32>(p, div, s);
        case 3208: return launch_forward_tu<32, 8>(p, div, s);
        case 801: return launch_forward_tu<8, 1>(p, div, s);
        case 804: return launch_forward_tu<8, 4>(p, div, s);
        default:
            set_error("unsupported forward-projector tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
}

int fp_launch_backward(const FpArgs& p, const FpTile& tile, bool gradvol, cudaStream_t s) {
    switch (tile.tu * 100 + tile.wu) {
        case 1608: return launch_backward_tu<16, 8>(p, gradvol, s);
        case 3232: return launch_backward_tu<32, 32>(p, gradvol, s);
        case 801: return launch_backward_tu<8, 1>(p, gradvol, s);
        default:
            set_error("unsupported backward tile");
            return DGC_ERR_INVALID_ARGUMENT;
    }
}

int fp_launch_counts(const FpArgs& p, int64_t* counts, cudaStream_t s) {
    DGC_TRACE("fp_count_kernel", s);
    const long long blocks = (long long)p.A * ceil_div(p.U, 16) * ceil_div(p.V, 16);
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
