// capi.cu -- extern "C" entry points of libdgc (see include/dgc.h).
//
// Argument checks reproduce the conditions of the reference's host wrappers
// (TomSHINING/diff-geoCali csrc/src_cbct_forwardprojector_cuda.cu:531-729 and
// csrc/src_cbct_backprojector_cuda.cu:298-522) with the same messages; a
// failed check returns DGC_ERR_INVALID_ARGUMENT, which the Python layer raises
// as RuntimeError exactly where the reference's TORCH_CHECK would.
#include <climits>
#include <cmath>
#include <cstdlib>
#include <string>

#include "backprojector.cuh"
#include "common.cuh"
#include "fdk.cuh"
#include "forward_projector.cuh"
#include "tc_gemm.cuh"

namespace dgc {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

namespace {

Geometry make_geometry(const float* angles, const float* sid, const float* sod,
                       const float* det_u0, const float* det_v0, const float* src_x,
                       const float* src_y, const float* src_z) {
    Geometry g;
    g.angles = angles;
    g.sid = sid;
    g.sod = sod;
    g.det_u0 = det_u0;
    g.det_v0 = det_v0;
    g.src_x = src_x;
    g.src_y = src_y;
    g.src_z = src_z;
    return g;
}

bool geometry_ok(const Geometry& g) {
    return g.angles && g.sid && g.sod && g.det_u0 && g.det_v0 && g.src_x && g.src_y && g.src_z;
}

size_t quad_volume_bytes(int D, int H, int W) {
    return Workspace::align(sizeof(float4) * (size_t)(D + 2) * (size_t)(H + 1) * (size_t)(W + 1));
}

// volume-gradient buffer (level records)
size_t gradient_buffer_bytes(int D, int H, int W) {
    return Workspace::align(sizeof(float) * fp_record_buffer_floats(D, H, W));
}

// Ray tile of the forward projector (8 detector columns x 32 rows per CTA):
// the batched launches take per-instance tiles from the autotuner.
constexpr FpTile kForwardTile{8, 1};
constexpr FpTile kBackwardTile{8, 1};

int check_fp_common(int D, int H, int W, int A, int U, int V, float pixel_size, float step_size,
                    float voxel_size, const Geometry& g) {
    DGC_REQUIRE(D > 0 && H > 0 && W > 0, "every volume dimension must be positive");
    DGC_REQUIRE(U > 0 && V > 0, "U and V must be positive");
    DGC_REQUIRE(pixel_size > 0.0f && step_size > 0.0f && voxel_size > 0.0f,
                "pixel_size, step_size and voxel_size must be positive");
    DGC_REQUIRE(A > 0, "angles must contain at least one view");
    DGC_REQUIRE(geometry_ok(g), "geometry pointers must be non-null");
    if ((long long)(D + 2) * (H + 1) * (W + 1) >= (1LL << 31)) {
        set_error("volume exceeds the library's 2^31 padded-voxel index limit");
        return DGC_ERR_UNSUPPORTED;
    }
    if (fp_tiles_per_view(U, V, 4) * (long long)A >= (1LL << 31)) {
        set_error("too many rays for one launch");
        return DGC_ERR_UNSUPPORTED;
    }
    return DGC_OK;
}

int check_bp_common(int A, int U, int V, int D, int H, int W, float pixel_size, float voxel_size,
                    float off_x, float off_y, float off_z, const Geometry& g) {
    DGC_REQUIRE(A > 0 && U >= 2 && V >= 2, "proj must have shape [A,U,V] with A >= 1 and U,V >= 2");
    DGC_REQUIRE((long long)A * U * V <= INT_MAX, "proj exceeds the kernel's 32-bit indexing limit");
    DGC_REQUIRE(D > 0 && H > 0 && W > 0, "D,H,W must be positive and fit in a 32-bit integer");
    DGC_REQUIRE((long long)D * H * W <= INT_MAX, "volume exceeds the kernel's 32-bit indexing limit");
    DGC_REQUIRE(D <= 8 * 65535 && H <= 8 * 65535, "D,H exceed the kernel's 3D CUDA grid limits");
    DGC_REQUIRE(std::isfinite(pixel_size) && std::isfinite(voxel_size) && std::isfinite(off_x) &&
                    std::isfinite(off_y) && std::isfinite(off_z),
                "sizes and ROI offsets must be finite");
    DGC_REQUIRE(pixel_size > 0.0f && voxel_size > 0.0f, "pixel_size and voxel_size must be positive");
    DGC_REQUIRE(geometry_ok(g), "geometry pointers must be non-null");
    return DGC_OK;
}

size_t bp_table_bytes(int A) { return Workspace::align(sizeof(ViewRow) * (size_t)A); }

size_t bp_quads_bytes(int A, int U, int V) {
    return Workspace::align(sizeof(float4) * (size_t)A * (size_t)(U - 1) * (size_t)(V - 1));
}

BpArgs bp_args(const ViewRow* vt, const float4* pq, int A, int U, int V, int D, int H, int W,
               float pixel_size, float voxel_size, float ox, float oy, float oz) {
    BpArgs p;
    memset(&p, 0, sizeof(p));
    p.vt = vt;
    p.pquads = pq;
    p.A = A;
    p.U = U;
    p.V = V;
    p.D = D;
    p.H = H;
    p.W = W;
    p.pixel_size = pixel_size;
    p.inv_pixel = 1.0f / pixel_size;
    p.voxel_size = voxel_size;
    p.off_x = ox;
    p.off_y = oy;
    p.off_z = oz;
    p.out_scale = 1.0f;
    p.clamp = 1;
    return p;
}

}  // namespace

int fp_check_args(int D, int H, int W, int A, int U, int V, float pixel_size, float step_size,
                  float voxel_size, const Geometry& g) {
    return check_fp_common(D, H, W, A, U, V, pixel_size, step_size, voxel_size, g);
}

}  // namespace dgc

using namespace dgc;

extern "C" {

int dgc_abi_version(void) { return DGC_ABI_VERSION; }

const char* dgc_last_error(void) { return g_last_error.c_str(); }

// ----------------------------------------------------------------- forward

size_t dgc_project_workspace_bytes(int D, int H, int W, int A, int U, int V) {
    (void)A;
    (void)U;
    (void)V;
    if (D <= 0 || H <= 0 || W <= 0) return 0;
    // the quad-packed volume and the status word of the TMA arm's bounded waits
    return quad_volume_bytes(D, H, W) + Workspace::align(sizeof(int));
}

static int project_impl(const float* volume, int D, int H, int W, const Geometry& g, int A,
                        float pixel_size, int U, int V, float step_size, float voxel_size,
                        float off_x, float off_y, float off_z, float* projections,
                        int64_t* counts, void* workspace, size_t workspace_bytes,
                        cudaStream_t s) {
    clear_error();
    int rc = check_fp_common(D, H, W, A, U, V, pixel_size, step_size, voxel_size, g);
    if (rc != DGC_OK) return rc;
    FpArgs p;
    memset(&p, 0, sizeof(p));
    p.g = g;
    p.D = D;
    p.H = H;
    p.W = W;
    p.A = A;
    p.U = U;
    p.V = V;
    p.pixel_size = pixel_size;
    p.step_size = step_size;
    p.voxel_size = voxel_size;
    p.off_x = off_x;
    p.off_y = off_y;
    p.off_z = off_z;
    fp_fill_layout(p);
    if (counts) return fp_launch_counts(p, counts, s);
    DGC_REQUIRE(volume && projections, "volume and projections must be non-null");
    Workspace ws(workspace, workspace_bytes);
    float4* quads = ws.take<float4>((size_t)(D + 2) * (H + 1) * (W + 1));
    int* status = ws.take<int>(1);
    if (!quads || !status) {
        set_error("workspace too small: dgc_project needs " +
                  std::to_string(dgc_project_workspace_bytes(D, H, W, A, U, V)) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    p.quads = quads;
    p.projections = projections;
    p.error = status;
    // the arm decided once: its layout is built into the quads' slice (the
    // z-pair layout is smaller)
    const FpArm arm = fp_forward_arm(D, H, W);
    rc = arm.arm == 2 ? build_volume_pairs(volume, D, H, W, reinterpret_cast<float2*>(quads), s)
                      : build_volume_quads(volume, D, H, W, quads, s);
    if (rc != DGC_OK) return rc;
    DGC_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    return fp_launch_forward(p, kForwardTile, arm, s);
}

int dgc_project(const float* volume, int D, int H, int W, const float* angles, const float* sid,
                const float* sod, const float* det_u0, const float* det_v0, const float* src_x,
                const float* src_y, const float* src_z, int A, float pixel_size, int U, int V,
                float step_size, float voxel_size, float off_x, float off_y, float off_z,
                float* projections, void* workspace, size_t workspace_bytes, void* stream) {
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    return project_impl(volume, D, H, W, g, A, pixel_size, U, V, step_size, voxel_size, off_x,
                        off_y, off_z, projections, nullptr, workspace, workspace_bytes,
                        (cudaStream_t)stream);
}

int dgc_project_sample_counts(int D, int H, int W, const float* angles, const float* sid,
                              const float* sod, const float* det_u0, const float* det_v0,
                              const float* src_x, const float* src_y, const float* src_z, int A,
                              float pixel_size, int U, int V, float step_size, float voxel_size,
                              float off_x, float off_y, float off_z, int64_t* counts,
                              void* stream) {
    if (!counts) {
        set_error("counts must be non-null");
        return DGC_ERR_INVALID_ARGUMENT;
    }
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    return project_impl(nullptr, D, H, W, g, A, pixel_size, U, V, step_size, voxel_size, off_x,
                        off_y, off_z, nullptr, counts, nullptr, 0, (cudaStream_t)stream);
}

size_t dgc_project_backward_workspace_bytes(int D, int H, int W, int A, int U, int V,
                                            int compute_grad_volume) {
    if (D <= 0 || H <= 0 || W <= 0 || A <= 0 || U <= 0 || V <= 0) return 0;
    size_t n = quad_volume_bytes(D, H, W);
    if (compute_grad_volume) n += gradient_buffer_bytes(D, H, W);
    n += Workspace::align(sizeof(double) * 8 * (size_t)A *
                          (size_t)fp_tiles_per_view(U, V, kBackwardTile.tu));
    return n;
}

int dgc_project_backward(const float* grad_projection, const float* volume, int D, int H, int W,
                         const float* angles, const float* sid, const float* sod,
                         const float* det_u0, const float* det_v0, const float* src_x,
                         const float* src_y, const float* src_z, int A, float pixel_size, int U,
                         int V, float step_size, float voxel_size, int compute_grad_volume,
                         float off_x, float off_y, float off_z, float* grad_volume,
                         float* grad_angles, float* grad_sid, float* grad_sod,
                         float* grad_det_u0, float* grad_det_v0, float* grad_src_x,
                         float* grad_src_y, float* grad_src_z, void* workspace,
                         size_t workspace_bytes, void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    int rc = check_fp_common(D, H, W, A, U, V, pixel_size, step_size, voxel_size, g);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(grad_projection && volume, "grad_projection and volume must be non-null");
    DGC_REQUIRE(!compute_grad_volume || grad_volume, "grad_volume must be non-null");
    GeometryGrad out{{grad_angles, grad_sid, grad_sod, grad_det_u0, grad_det_v0, grad_src_x,
                      grad_src_y, grad_src_z}};
    for (int k = 0; k < 8; ++k) DGC_REQUIRE(out.g[k], "geometry gradient pointers must be non-null");
    FpArgs p;
    memset(&p, 0, sizeof(p));
    p.g = g;
    p.D = D;
    p.H = H;
    p.W = W;
    p.A = A;
    p.U = U;
    p.V = V;
    p.pixel_size = pixel_size;
    p.step_size = step_size;
    p.voxel_size = voxel_size;
    p.off_x = off_x;
    p.off_y = off_y;
    p.off_z = off_z;
    fp_fill_layout(p);
    const long long tiles = fp_tiles_per_view(U, V, kBackwardTile.tu);
    Workspace ws(workspace, workspace_bytes);
    float4* quads = ws.take<float4>((size_t)(D + 2) * (H + 1) * (W + 1));
    const size_t gfloats = fp_record_buffer_floats(D, H, W);
    float* gpad = compute_grad_volume ? ws.take<float>(gfloats) : nullptr;
    double* partials = ws.take<double>((size_t)8 * A * tiles);
    if (!quads || !partials || (compute_grad_volume && !gpad)) {
        set_error("workspace too small: dgc_project_backward needs " +
                  std::to_string(dgc_project_backward_workspace_bytes(D, H, W, A, U, V,
                                                                      compute_grad_volume)) +
                  " bytes");
        return DGC_ERR_WORKSPACE;
    }
    p.quads = quads;
    p.grad_projections = grad_projection;
    p.grad_pad = gpad;
    p.partials = partials;
    rc = build_volume_quads(volume, D, H, W, quads, s);
    if (rc != DGC_OK) return rc;
    if (gpad) DGC_CUDA(cudaMemsetAsync(gpad, 0, sizeof(float) * gfloats, s));
    rc = fp_launch_backward(p, kBackwardTile, compute_grad_volume != 0, s);
    if (rc != DGC_OK) return rc;
    rc = fp_reduce_partials(partials, A, tiles, out, s);
    if (rc != DGC_OK) return rc;
    if (gpad) return fp_fold_records(gpad, D, H, W, grad_volume, s);
    return DGC_OK;
}

// ------------------------------------------- fused calibration loss + grads

size_t dgc_project_mse_grad_workspace_bytes(int D, int H, int W, int A, int U, int V) {
    if (D <= 0 || H <= 0 || W <= 0 || A <= 0 || U <= 0 || V <= 0) return 0;
    const size_t tiles = (size_t)fp_tiles_per_view(U, V, fp_mse_tile(D, H, W)) * (size_t)A;
    return quad_volume_bytes(D, H, W) + Workspace::align(sizeof(double) * 8 * tiles) +
           Workspace::align(sizeof(double) * tiles);
}

int dgc_project_mse_grad(const float* volume, int D, int H, int W, const float* angles,
                         const float* sid, const float* sod, const float* det_u0,
                         const float* det_v0, const float* src_x, const float* src_y,
                         const float* src_z, int A, float pixel_size, int U, int V,
                         float step_size, float voxel_size, float off_x, float off_y, float off_z,
                         const float* measured, const float* mask, float scale,
                         float* projections, double* loss, float* grad_angles, float* grad_sid,
                         float* grad_sod, float* grad_det_u0, float* grad_det_v0,
                         float* grad_src_x, float* grad_src_y, float* grad_src_z,
                         void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    int rc = check_fp_common(D, H, W, A, U, V, pixel_size, step_size, voxel_size, g);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(volume && measured && loss, "volume, measured and loss must be non-null");
    DGC_REQUIRE(std::isfinite(scale), "scale must be finite");
    GeometryGrad out{{grad_angles, grad_sid, grad_sod, grad_det_u0, grad_det_v0, grad_src_x,
                      grad_src_y, grad_src_z}};
    for (int k = 0; k < 8; ++k) DGC_REQUIRE(out.g[k], "geometry gradient pointers must be non-null");
    FpArgs p;
    memset(&p, 0, sizeof(p));
    p.g = g;
    p.D = D;
    p.H = H;
    p.W = W;
    p.A = A;
    p.U = U;
    p.V = V;
    p.pixel_size = pixel_size;
    p.step_size = step_size;
    p.voxel_size = voxel_size;
    p.off_x = off_x;
    p.off_y = off_y;
    p.off_z = off_z;
    fp_fill_layout(p);
    const int tile = fp_mse_tile(D, H, W);
    const long long tiles = fp_tiles_per_view(U, V, tile);
    Workspace ws(workspace, workspace_bytes);
    float4* quads = ws.take<float4>((size_t)(D + 2) * (H + 1) * (W + 1));
    double* partials = ws.take<double>((size_t)8 * A * tiles);
    double* lpart = ws.take<double>((size_t)A * tiles);
    if (!quads || !partials || !lpart) {
        set_error("workspace too small: dgc_project_mse_grad needs " +
                  std::to_string(dgc_project_mse_grad_workspace_bytes(D, H, W, A, U, V)) +
                  " bytes");
        return DGC_ERR_WORKSPACE;
    }
    p.quads = quads;
    p.partials = partials;
    p.projections = projections;
    // the forward's CTA order for this volume (the fused step marches the same rays)
    p.view_block = fp_forward_arm(D, H, W).view_block;
    rc = build_volume_quads(volume, D, H, W, quads, s);
    if (rc != DGC_OK) return rc;
    rc = fp_launch_mse_grad(p, tile, measured, mask, scale, lpart, s);
    if (rc != DGC_OK) return rc;
    rc = fp_reduce_partials(partials, A, tiles, out, s);
    if (rc != DGC_OK) return rc;
    return fp_sum_partials(lpart, (long long)A * tiles, (double)scale, loss, s);
}

// ----------------------------------------------------------- backprojector

size_t dgc_backproject_workspace_bytes(int A, int U, int V, int D, int H, int W) {
    (void)D;
    (void)H;
    (void)W;
    if (A <= 0 || U < 2 || V < 2) return 0;
    return bp_table_bytes(A) + bp_quads_bytes(A, U, V);
}

int dgc_backproject(const float* projections, int A, int U, int V, const float* angles,
                    const float* sid, const float* sod, const float* det_u0, const float* det_v0,
                    const float* src_x, const float* src_y, const float* src_z, float pixel_size,
                    int D, int H, int W, float voxel_size, float off_x, float off_y, float off_z,
                    float* volume, void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    int rc = check_bp_common(A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z, g);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(projections && volume, "projections and volume must be non-null");
    Workspace ws(workspace, workspace_bytes);
    ViewRow* vt = ws.take<ViewRow>((size_t)A);
    float4* pq = ws.take<float4>((size_t)A * (U - 1) * (V - 1));
    if (!vt || !pq) {
        set_error("workspace too small: dgc_backproject needs " +
                  std::to_string(dgc_backproject_workspace_bytes(A, U, V, D, H, W)) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    if ((rc = bp_view_table(g, A, vt, s)) != DGC_OK) return rc;
    if ((rc = build_proj_quads(projections, A, U, V, pq, s)) != DGC_OK) return rc;
    BpArgs p = bp_args(vt, pq, A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z);
    p.volume = volume;
    return bp_launch_forward(p, false, s);
}

size_t dgc_backproject_backward_workspace_bytes(int A, int U, int V, int D, int H, int W) {
    if (A <= 0 || U < 2 || V < 2 || D <= 0 || H <= 0 || W <= 0) return 0;
    return bp_table_bytes(A) + bp_quads_bytes(A, U, V) +
           Workspace::align(sizeof(double) * 8 * (size_t)A * (size_t)bp_backward_blocks(D, H, W, bp_kz_backward(D, A)));
}

int dgc_backproject_backward(const float* grad_volume, const float* projections, int A, int U,
                             int V, const float* angles, const float* sid, const float* sod,
                             const float* det_u0, const float* det_v0, const float* src_x,
                             const float* src_y, const float* src_z, float pixel_size, int D,
                             int H, int W, float voxel_size, float off_x, float off_y,
                             float off_z, float* grad_projections, float* grad_angles,
                             float* grad_sid, float* grad_sod, float* grad_det_u0,
                             float* grad_det_v0, float* grad_src_x, float* grad_src_y,
                             float* grad_src_z, void* workspace, size_t workspace_bytes,
                             void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    int rc = check_bp_common(A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z, g);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(grad_volume && projections, "grad_vol and proj must be non-null");
    GeometryGrad out{{grad_angles, grad_sid, grad_sod, grad_det_u0, grad_det_v0, grad_src_x,
                      grad_src_y, grad_src_z}};
    for (int k = 0; k < 8; ++k) DGC_REQUIRE(out.g[k], "geometry gradient pointers must be non-null");
    const int kz = bp_kz_backward(D, A);
    const long long nblocks = bp_backward_blocks(D, H, W, kz);
    Workspace ws(workspace, workspace_bytes);
    ViewRow* vt = ws.take<ViewRow>((size_t)A);
    float4* pq = ws.take<float4>((size_t)A * (U - 1) * (V - 1));
    double* partials = ws.take<double>((size_t)8 * A * nblocks);
    if (!vt || !pq || !partials) {
        set_error("workspace too small: dgc_backproject_backward needs " +
                  std::to_string(dgc_backproject_backward_workspace_bytes(A, U, V, D, H, W)) +
                  " bytes");
        return DGC_ERR_WORKSPACE;
    }
    if ((rc = bp_view_table(g, A, vt, s)) != DGC_OK) return rc;
    if ((rc = build_proj_quads(projections, A, U, V, pq, s)) != DGC_OK) return rc;
    BpArgs p = bp_args(vt, pq, A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z);
    if (grad_projections) {
        DGC_CUDA(cudaMemsetAsync(grad_projections, 0, sizeof(float) * (size_t)A * U * V, s));
        p.grad_projections = grad_projections;
    }
    p.grad_volume = grad_volume;
    p.partials = partials;
    p.kz_backward = kz;
    if ((rc = bp_launch_backward(p, s)) != DGC_OK) return rc;
    return bp_reduce_partials(partials, A, nblocks, out, s);
}

// --------------------------------------------------------------------- FDK

int dgc_fdk_filter_taps(int U, double pixel_size, double alpha, double* taps) {
    clear_error();
    DGC_REQUIRE(U > 0 && taps, "U must be positive and taps non-null");
    DGC_REQUIRE(std::isfinite(pixel_size) && pixel_size > 0.0, "pixel_size must be finite and positive");
    DGC_REQUIRE(std::isfinite(alpha) && alpha > 0.0 && alpha <= 1.0, "alpha must satisfy 0 < alpha <= 1");
    std::vector<double> h;
    int rc = fdk_taps_host(U, pixel_size, alpha, h);
    if (rc != DGC_OK) return rc;
    for (int i = 0; i < U; ++i) taps[i] = h[i];
    return DGC_OK;
}

size_t dgc_fdk_filter_workspace_bytes(int A, int U, int V) {
    (void)A;
    (void)V;
    if (U <= 0) return 0;
    return Workspace::align(sizeof(float) * (size_t)U);
}

static int check_fdk(int A, int U, int V, float pixel_size, float alpha) {
    DGC_REQUIRE(A > 0 && U > 0 && V > 0, "projections must have a nonempty [A, U, V] shape");
    DGC_REQUIRE(std::isfinite(pixel_size) && pixel_size > 0.0f, "pixel_size must be finite and positive");
    DGC_REQUIRE(std::isfinite(alpha) && alpha > 0.0f, "alpha must be finite and positive");
    DGC_REQUIRE(alpha <= 1.0f, "alpha must satisfy 0 < alpha <= 1");
    return DGC_OK;
}

int dgc_fdk_filter_ex(const float* projections, int A, int U, int V, float pixel_size,
                      const float* sod, const float* sid, const float* frame_dist,
                      const float* frame_u, const float* frame_v, float alpha, float* filtered,
                      void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    int rc = check_fdk(A, U, V, pixel_size, alpha);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(projections && sod && sid && filtered, "pointers must be non-null");
    Workspace ws(workspace, workspace_bytes);
    float* taps = ws.take<float>((size_t)U);
    if (!taps) {
        set_error("workspace too small: dgc_fdk_filter needs " +
                  std::to_string(dgc_fdk_filter_workspace_bytes(A, U, V)) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    if ((rc = fdk_upload_taps(U, pixel_size, alpha, taps, s)) != DGC_OK) return rc;
    FdkArgs f{projections, sod, sid, taps, filtered, A, U, V, pixel_size};
    f.frame_dist = frame_dist;
    f.frame_u = frame_u;
    f.frame_v = frame_v;
    return fdk_launch_filter(f, s);
}

int dgc_fdk_filter(const float* projections, int A, int U, int V, float pixel_size,
                   const float* sod, const float* sid, float alpha, float* filtered,
                   void* workspace, size_t workspace_bytes, void* stream) {
    return dgc_fdk_filter_ex(projections, A, U, V, pixel_size, sod, sid, nullptr, nullptr, nullptr,
                             alpha, filtered, workspace, workspace_bytes, stream);
}

size_t dgc_fdk_filter_backward_workspace_bytes(int A, int U, int V) {
    if (A <= 0 || U <= 0 || V <= 0) return 0;
    return Workspace::align(sizeof(float) * (size_t)U) +
           Workspace::align(sizeof(double) * kFdkPartials * (size_t)A *
                            (size_t)fdk_filter_tiles(U, V));
}

int dgc_fdk_filter_backward_ex(const float* grad_filtered, const float* projections,
                               const float* filtered, int A, int U, int V, float pixel_size,
                               const float* sod, const float* sid, const float* frame_dist,
                               const float* frame_u, const float* frame_v, float alpha,
                               float* grad_projections, float* grad_sod, float* grad_sid,
                               float* grad_frame_dist, float* grad_frame_u, float* grad_frame_v,
                               void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    int rc = check_fdk(A, U, V, pixel_size, alpha);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(grad_filtered && sod && sid, "grad_filtered, sod and sid must be non-null");
    DGC_REQUIRE((!grad_frame_dist || frame_dist) && (!grad_frame_u || frame_u) &&
                    (!grad_frame_v || frame_v),
                "a frame gradient needs the frame array it belongs to");
    const bool dist = grad_sod || grad_sid || grad_frame_dist || grad_frame_u || grad_frame_v;
    DGC_REQUIRE(!dist || (projections && filtered),
                "the distance and frame gradients need projections and filtered");
    if (!grad_projections && !dist) return DGC_OK;
    const long long tiles = fdk_filter_tiles(U, V);
    Workspace ws(workspace, workspace_bytes);
    float* taps = ws.take<float>((size_t)U);
    double* partials = ws.take<double>((size_t)kFdkPartials * A * tiles);
    if (!taps || !partials) {
        set_error("workspace too small: dgc_fdk_filter_backward needs " +
                  std::to_string(dgc_fdk_filter_backward_workspace_bytes(A, U, V)) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    if ((rc = fdk_upload_taps(U, pixel_size, alpha, taps, s)) != DGC_OK) return rc;
    FdkArgs f{projections, sod, sid, taps, nullptr, A, U, V, pixel_size};
    f.grad_filtered = grad_filtered;
    f.forward_out = filtered;
    f.grad_projections = grad_projections;
    f.partials = dist ? partials : nullptr;
    f.frame_dist = frame_dist;
    f.frame_u = frame_u;
    f.frame_v = frame_v;
    f.frame_grads = (grad_frame_u || grad_frame_v) ? 1 : 0;
    if ((rc = fdk_launch_filter_adjoint(f, s)) != DGC_OK) return rc;
    if (!dist) return DGC_OK;
    const FdkGrads g{grad_sod, grad_sid, grad_frame_dist, grad_frame_u, grad_frame_v};
    return fdk_reduce_distance_grads(partials, A, tiles, f, g, s);
}

int dgc_fdk_filter_backward(const float* grad_filtered, const float* projections,
                            const float* filtered, int A, int U, int V, float pixel_size,
                            const float* sod, const float* sid, float alpha,
                            float* grad_projections, float* grad_sod, float* grad_sid,
                            void* workspace, size_t workspace_bytes, void* stream) {
    return dgc_fdk_filter_backward_ex(grad_filtered, projections, filtered, A, U, V, pixel_size,
                                      sod, sid, nullptr, nullptr, nullptr, alpha,
                                      grad_projections, grad_sod, grad_sid, nullptr, nullptr,
                                      nullptr, workspace, workspace_bytes, stream);
}

size_t dgc_reconstruct_fdk_workspace_bytes(int A, int U, int V, int D, int H, int W) {
    if (A <= 0 || U < 2 || V < 2) return 0;
    return dgc_fdk_filter_workspace_bytes(A, U, V) +
           Workspace::align(sizeof(float) * (size_t)A * U * V) +
           dgc_backproject_workspace_bytes(A, U, V, D, H, W);
}

static int reconstruct_fdk_impl(const float* projections, int A, int U, int V,
                                const float* angles, const float* sid, const float* sod,
                                const float* det_u0, const float* det_v0, const float* src_x,
                                const float* src_y, const float* src_z, float pixel_size, int D,
                                int H, int W, float voxel_size, float off_x, float off_y,
                                float off_z, float alpha, const float* frame_dist,
                                const float* frame_u, const float* frame_v,
                                const float* uweights, float angle_scale, bool clamp,
                                float* volume, void* workspace, size_t workspace_bytes,
                                void* stream) {
    clear_error();
    cudaStream_t s = (cudaStream_t)stream;
    const Geometry g = make_geometry(angles, sid, sod, det_u0, det_v0, src_x, src_y, src_z);
    int rc = check_fdk(A, U, V, pixel_size, alpha);
    if (rc != DGC_OK) return rc;
    rc = check_bp_common(A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z, g);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(projections && volume, "projections and volume must be non-null");
    Workspace ws(workspace, workspace_bytes);
    float* taps = ws.take<float>((size_t)U);
    float* filtered = ws.take<float>((size_t)A * U * V);
    ViewRow* vt = ws.take<ViewRow>((size_t)A);
    float4* pq = ws.take<float4>((size_t)A * (U - 1) * (V - 1));
    if (!taps || !filtered || !vt || !pq) {
        set_error("workspace too small: dgc_reconstruct_fdk needs " +
                  std::to_string(dgc_reconstruct_fdk_workspace_bytes(A, U, V, D, H, W)) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    if ((rc = fdk_upload_taps(U, pixel_size, alpha, taps, s)) != DGC_OK) return rc;
    FdkArgs f{projections, sod, sid, taps, filtered, A, U, V, pixel_size, uweights};
    f.frame_dist = frame_dist;
    f.frame_u = frame_u;
    f.frame_v = frame_v;
    if ((rc = fdk_launch_filter(f, s)) != DGC_OK) return rc;
    if ((rc = bp_view_table(g, A, vt, s)) != DGC_OK) return rc;
    if ((rc = build_proj_quads(filtered, A, U, V, pq, s)) != DGC_OK) return rc;
    BpArgs p = bp_args(vt, pq, A, U, V, D, H, W, pixel_size, voxel_size, off_x, off_y, off_z);
    p.volume = volume;
    p.out_scale = angle_scale;
    p.clamp = clamp ? 1 : 0;
    return bp_launch_forward(p, true, s);
}

int dgc_reconstruct_fdk(const float* projections, int A, int U, int V, const float* angles,
                        const float* sid, const float* sod, const float* det_u0,
                        const float* det_v0, const float* src_x, const float* src_y,
                        const float* src_z, float pixel_size, int D, int H, int W,
                        float voxel_size, float off_x, float off_y, float off_z, float alpha,
                        float* volume, void* workspace, size_t workspace_bytes, void* stream) {
    return reconstruct_fdk_impl(projections, A, U, V, angles, sid, sod, det_u0, det_v0, src_x,
                                src_y, src_z, pixel_size, D, H, W, voxel_size, off_x, off_y, off_z,
                                alpha, nullptr, nullptr, nullptr, nullptr,
                                (float)(M_PI / (double)A), true, volume, workspace,
                                workspace_bytes, stream);
}

int dgc_reconstruct_fdk_weighted(const float* projections, int A, int U, int V,
                                 const float* angles, const float* sid, const float* sod,
                                 const float* det_u0, const float* det_v0, const float* src_x,
                                 const float* src_y, const float* src_z, float pixel_size, int D,
                                 int H, int W, float voxel_size, float off_x, float off_y,
                                 float off_z, float alpha, const float* uweights,
                                 float angle_scale, float* volume, void* workspace,
                                 size_t workspace_bytes, void* stream) {
    clear_error();
    DGC_REQUIRE(std::isfinite(angle_scale) && angle_scale > 0.0f,
                "angle_scale must be positive and finite");
    return reconstruct_fdk_impl(projections, A, U, V, angles, sid, sod, det_u0, det_v0, src_x,
                                src_y, src_z, pixel_size, D, H, W, voxel_size, off_x, off_y, off_z,
                                alpha, nullptr, nullptr, nullptr, uweights, angle_scale, true,
                                volume, workspace, workspace_bytes, stream);
}

int dgc_reconstruct_fdk_partial(const float* projections, int A, int U, int V,
                                const float* angles, const float* sid, const float* sod,
                                const float* det_u0, const float* det_v0, const float* src_x,
                                const float* src_y, const float* src_z, float pixel_size, int D,
                                int H, int W, float voxel_size, float off_x, float off_y,
                                float off_z, float alpha, const float* uweights,
                                float angle_scale, float* volume, void* workspace,
                                size_t workspace_bytes, void* stream) {
    clear_error();
    DGC_REQUIRE(std::isfinite(angle_scale) && angle_scale > 0.0f,
                "angle_scale must be positive and finite");
    return reconstruct_fdk_impl(projections, A, U, V, angles, sid, sod, det_u0, det_v0, src_x,
                                src_y, src_z, pixel_size, D, H, W, voxel_size, off_x, off_y, off_z,
                                alpha, nullptr, nullptr, nullptr, uweights, angle_scale, false,
                                volume, workspace, workspace_bytes, stream);
}

int dgc_reconstruct_fdk_ex(const float* projections, int A, int U, int V, const float* angles,
                           const float* sid, const float* sod, const float* det_u0,
                           const float* det_v0, const float* src_x, const float* src_y,
                           const float* src_z, float pixel_size, int D, int H, int W,
                           float voxel_size, float off_x, float off_y, float off_z, float alpha,
                           const float* frame_dist, const float* frame_u, const float* frame_v,
                           const float* uweights, float angle_scale, int clamp, float* volume,
                           void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    DGC_REQUIRE(std::isfinite(angle_scale) && angle_scale > 0.0f,
                "angle_scale must be positive and finite");
    return reconstruct_fdk_impl(projections, A, U, V, angles, sid, sod, det_u0, det_v0, src_x,
                                src_y, src_z, pixel_size, D, H, W, voxel_size, off_x, off_y, off_z,
                                alpha, frame_dist, frame_u, frame_v, uweights, angle_scale,
                                clamp != 0, volume, workspace, workspace_bytes, stream);
}

int dgc_bp_add_tile_rule(int d_max, int a_max, int kz_forward, int kz_backward, int cta_x,
                         int cta_y) {
    clear_error();
    const int rc = bp_add_tile_rule(d_max, a_max, kz_forward, kz_backward, cta_x, cta_y);
    if (rc == -2) {
        set_error("dgc_bp_add_tile_rule: the rule table is full");
        return DGC_ERR_INVALID_ARGUMENT;
    }
    DGC_REQUIRE(rc == 0, "dgc_bp_add_tile_rule: need d_max, a_max >= 1, kz in {0,1,2,4,8} and "
                         "cta_x = cta_y = 0 or cta_x, cta_y >= 1 with cta_x*cta_y <= 16");
    return DGC_OK;
}

int dgc_bp_clear_tile_rules(void) {
    clear_error();
    bp_clear_tile_rules();
    return DGC_OK;
}

int dgc_bp_tiles(int D, int A, int* kz_forward, int* kz_backward, int* cta_x, int* cta_y) {
    clear_error();
    DGC_REQUIRE(D >= 1 && A >= 1, "D and A must be positive");
    DGC_REQUIRE(kz_forward && kz_backward && cta_x && cta_y, "output pointers must be non-null");
    *kz_forward = bp_kz_forward(D, A);
    *kz_backward = bp_kz_backward(D, A);
    bp_forward_cta(D, A, *cta_x, *cta_y);
    return DGC_OK;
}

int dgc_fp_add_arm_rule(long long voxels_max, int arm, int slab_cells, int unroll,
                        int view_block) {
    using namespace dgc;
    clear_error();
    const int rc = fp_add_arm_rule(voxels_max, arm, slab_cells, unroll, view_block);
    if (rc == -2) {
        set_error("dgc_fp_add_arm_rule: the rule table is full");
        return DGC_ERR_UNSUPPORTED;
    }
    DGC_REQUIRE(rc == 0, "dgc_fp_add_arm_rule: need voxels_max >= 1, arm 0 (L1) or 1 (TMA), "
                         "for arm 1 slab_cells 2 or 4, unroll 1 or 2 (arm 1: 1), "
                         "0 <= view_block <= 65535");
    return DGC_OK;
}

int dgc_fp_clear_arm_rules(void) {
    dgc::clear_error();
    dgc::fp_clear_arm_rules();
    return DGC_OK;
}

int dgc_fp_arm(int D, int H, int W, int* arm, int* slab_cells, int* unroll, int* view_block) {
    using namespace dgc;
    clear_error();
    DGC_REQUIRE(arm && slab_cells && unroll && view_block, "pointers must be non-null");
    fp_forward_arm(D, H, W, arm, slab_cells, unroll, view_block);
    return DGC_OK;
}

int dgc_clamp_volume(float* volume, long long n, void* stream) {
    clear_error();
    DGC_REQUIRE(n >= 0, "n must be non-negative");
    DGC_REQUIRE(volume || n == 0, "volume must be non-null");
    if (n == 0) return DGC_OK;
    return bp_clamp_volume(volume, n, (cudaStream_t)stream);
}

int dgc_parker_weights_ex(const float* angles, const float* sid, const float* frame_dist,
                          const float* frame_u, int A, int U, float pixel_size, float* weights,
                          void* stream) {
    clear_error();
    DGC_REQUIRE(angles && sid && weights, "angles, sid and weights must be non-null");
    DGC_REQUIRE(A >= 2 && U >= 1, "a short scan needs A >= 2 views and U >= 1");
    DGC_REQUIRE((long long)A * U <= INT_MAX, "A*U exceeds the 32-bit launch limit");
    DGC_REQUIRE(std::isfinite(pixel_size) && pixel_size > 0.0f, "pixel_size must be positive");
    return fdk_parker_weights(angles, sid, frame_dist, frame_u, A, U, pixel_size, weights,
                              (cudaStream_t)stream);
}

int dgc_parker_weights(const float* angles, const float* sid, int A, int U, float pixel_size,
                       float* weights, void* stream) {
    return dgc_parker_weights_ex(angles, sid, nullptr, nullptr, A, U, pixel_size, weights, stream);
}

// ---------------------------------------------------------- tensor-core GEMM

int dgc_gemm_bf16(const void* A, const void* B, void* C, const float* bias, int M, int N, int K,
                  int lda, int ldb, int ldc, int c_bf16, int relu, int accumulate, float alpha,
                  int* error_flag, void* stream) {
    clear_error();
    DGC_REQUIRE(A && B && C && error_flag, "A, B, C and error_flag must be non-null");
    DGC_REQUIRE(M > 0 && N > 0 && K > 0, "M, N, K must be positive");
    DGC_REQUIRE(K % 8 == 0 && lda % 8 == 0 && ldb % 8 == 0 && lda >= K && ldb >= K,
                "K, lda and ldb must be multiples of 8 (16-byte rows) with lda, ldb >= K");
    DGC_REQUIRE(ldc >= N, "ldc must be >= N");
    DGC_REQUIRE(((uintptr_t)A % 16) == 0 && ((uintptr_t)B % 16) == 0,
                "A and B must be 16-byte aligned");
    DGC_REQUIRE(!(accumulate && c_bf16), "accumulate needs an fp32 C");
    DGC_REQUIRE(ceil_div(M, 128) <= 65535, "M too large for one launch");
    GemmArgs p{static_cast<const __nv_bfloat16*>(A), static_cast<const __nv_bfloat16*>(B), C, bias,
               M, N, K, lda, ldb, ldc, c_bf16, relu, accumulate, alpha, error_flag, 0};
    // Long reductions with few output tiles (weight gradients): split K over
    // CTAs and sum into a zeroed fp32 C with atomics.
    const long long tiles = (long long)ceil_div(M, 128) * ceil_div(N, N <= 64 ? 64 : 128);
    const int ktiles = ceil_div(K, 64);
    if (!c_bf16 && !relu && tiles < 148 && ktiles >= 32) {
        const int splits = (int)std::min<long long>(std::max<long long>(296 / tiles, 1), ktiles / 8);
        if (splits > 1) {
            p.k_tiles_per_split = ceil_div(ktiles, splits);
            // zero only the M x N window: C may be a column slice of a wider array
            if (!accumulate)
                DGC_CUDA(cudaMemset2DAsync(C, sizeof(float) * (size_t)ldc, 0, sizeof(float) * (size_t)N,
                                           (size_t)M, (cudaStream_t)stream));
        }
    }
    return tc_gemm(p, (cudaStream_t)stream);
}

}  // extern "C"
