// batch.cu -- host side of the batched forward projection / backward: plan a
// set of uneven instances into one caller-owned workspace and launch them as
// a handful of kernels (see the batched kernels in forward_projector.cu).
// No counterpart in the reference, which runs one problem per call.
//
// Workspace layout (256-byte aligned slices):
//   BatchInstance[n] | item_fwd[n+1] | item_bwd[n+1] | quad_block[n+1] |
//   view[n+1] | fold_block[n+1] | counters[2] |
//   per instance: quads | partials            | ... |
//   per instance with a volume gradient: gradient buffer | ...
// (level records).  The gradient buffers are contiguous, so one memset
// clears all of them.
#include <string>
#include <vector>

#include "common.cuh"
#include "forward_projector.cuh"

namespace dgc {
namespace {

size_t align256(size_t n) { return Workspace::align(n); }

size_t quads_bytes(const dgc_fp_instance& in) {
    return align256(sizeof(float4) * (size_t)(in.D + 2) * (size_t)(in.H + 1) * (size_t)(in.W + 1));
}

// volume-gradient buffer (level records)
size_t gpad_bytes(const dgc_fp_instance& in) {
    return align256(sizeof(float) * fp_record_buffer_floats(in.D, in.H, in.W));
}

int tile_fwd(const dgc_fp_instance& in) { return in.tile_forward == 0 ? 8 : in.tile_forward; }
int tile_bwd(const dgc_fp_instance& in) { return in.tile_backward == 0 ? 8 : in.tile_backward; }

size_t partials_bytes(const dgc_fp_instance& in) {
    return align256(sizeof(double) * 8 * (size_t)in.A *
                    (size_t)fp_tiles_per_view(in.U, in.V, tile_bwd(in)));
}

size_t tables_bytes(int n) {
    return align256(sizeof(BatchInstance) * (size_t)n) +
           5 * align256(sizeof(long long) * (size_t)(n + 1)) + align256(2 * sizeof(unsigned long long));
}

Geometry geometry_of(const dgc_fp_instance& in) {
    Geometry g;
    g.angles = in.angles;
    g.sid = in.sid;
    g.sod = in.sod;
    g.det_u0 = in.det_u0;
    g.det_v0 = in.det_v0;
    g.src_x = in.src_x;
    g.src_y = in.src_y;
    g.src_z = in.src_z;
    return g;
}

BatchTables tables_at(void* workspace, int n) {
    char* base = static_cast<char*>(workspace);
    BatchTables t;
    size_t off = 0;
    t.inst = reinterpret_cast<const BatchInstance*>(base);
    off += align256(sizeof(BatchInstance) * (size_t)n);
    const long long** arrays[5] = {&t.item_fwd, &t.item_bwd, &t.quad_block, &t.view, &t.fold_block};
    for (auto a : arrays) {
        *a = reinterpret_cast<const long long*>(base + off);
        off += align256(sizeof(long long) * (size_t)(n + 1));
    }
    t.counters = reinterpret_cast<unsigned long long*>(base + off);
    t.n = n;
    return t;
}

int check_instance(const dgc_fp_instance& in, int index) {
    const std::string where = "instance " + std::to_string(index) + ": ";
    const int rc = fp_check_args(in.D, in.H, in.W, in.A, in.U, in.V, in.pixel_size, in.step_size,
                                 in.voxel_size, geometry_of(in));
    if (rc != DGC_OK) {
        set_error(where + dgc_last_error());
        return rc;
    }
    DGC_REQUIRE(in.volume && in.projections, where + "volume and projections must be non-null");
    DGC_REQUIRE(in.tile_forward == 0 || in.tile_forward == 8 || in.tile_forward == 4 ||
                    in.tile_forward == 2,
                where + "tile_forward must be 0, 8, 4 or 2");
    DGC_REQUIRE(in.tile_backward == 0 || in.tile_backward == 8 || in.tile_backward == 4,
                where + "tile_backward must be 0, 8 or 4");
    return DGC_OK;
}

}  // namespace
}  // namespace dgc

using namespace dgc;

extern "C" {

size_t dgc_batch_workspace_bytes(const dgc_fp_instance* instances, int n) {
    if (!instances || n <= 0) return 0;
    size_t bytes = tables_bytes(n);
    for (int i = 0; i < n; ++i) {
        const dgc_fp_instance& in = instances[i];
        if (in.D <= 0 || in.H <= 0 || in.W <= 0 || in.A <= 0 || in.U <= 0 || in.V <= 0) return 0;
        bytes += quads_bytes(in) + partials_bytes(in);
        if (in.grad_volume) bytes += gpad_bytes(in);
    }
    return bytes;
}

int dgc_batch_prepare(const dgc_fp_instance* instances, int n, void* workspace,
                      size_t workspace_bytes, dgc_batch_plan* plan, void* stream) {
    clear_error();
    DGC_REQUIRE(instances && n > 0, "a batch needs at least one instance");
    DGC_REQUIRE(plan, "plan must be non-null");
    for (int i = 0; i < n; ++i) {
        const int rc = check_instance(instances[i], i);
        if (rc != DGC_OK) return rc;
    }
    const size_t need = dgc_batch_workspace_bytes(instances, n);
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255u)) {
        set_error("workspace too small or not 256-byte aligned: dgc_batch_prepare needs " +
                  std::to_string(need) + " bytes");
        return DGC_ERR_WORKSPACE;
    }
    char* base = static_cast<char*>(workspace);
    const size_t tb = tables_bytes(n);
    size_t off = tb;
    size_t gpad_total = 0;
    for (int i = 0; i < n; ++i) off += quads_bytes(instances[i]) + partials_bytes(instances[i]);
    const size_t gpad_off = off;

    std::vector<BatchInstance> host(n);
    std::vector<long long> prefix(5 * (size_t)(n + 1), 0);
    long long* item_fwd = prefix.data();
    long long* item_bwd = item_fwd + (n + 1);
    long long* quad_block = item_bwd + (n + 1);
    long long* view = quad_block + (n + 1);
    long long* fold_block = view + (n + 1);
    long long rays = 0;
    int backward_ready = 1;
    size_t inst_off = tb;
    for (int i = 0; i < n; ++i) {
        const dgc_fp_instance& in = instances[i];
        BatchInstance b;
        memset(&b, 0, sizeof(b));
        FpArgs& p = b.p;
        p.g = geometry_of(in);
        p.D = in.D;
        p.H = in.H;
        p.W = in.W;
        p.A = in.A;
        p.U = in.U;
        p.V = in.V;
        p.pixel_size = in.pixel_size;
        p.step_size = in.step_size;
        p.voxel_size = in.voxel_size;
        p.off_x = in.off_x;
        p.off_y = in.off_y;
        p.off_z = in.off_z;
        fp_fill_layout(p);
        p.quads = reinterpret_cast<const float4*>(base + inst_off);
        inst_off += quads_bytes(in);
        p.partials = reinterpret_cast<double*>(base + inst_off);
        inst_off += partials_bytes(in);
        p.projections = in.projections;
        p.grad_projections = in.grad_projections;
        if (in.grad_volume) {
            p.grad_pad = reinterpret_cast<float*>(base + gpad_off + gpad_total);
            gpad_total += gpad_bytes(in);
        }
        b.volume = in.volume;
        b.grad_volume = in.grad_volume;
        for (int k = 0; k < 8; ++k)
            b.gout.g[k] = in.grad_geometry ? in.grad_geometry + (size_t)k * in.A : nullptr;
        b.tile_fwd = tile_fwd(in);
        b.tile_bwd = tile_bwd(in);
        b.flags = (is_pow2_float(in.voxel_size) ? 0 : kBatchDiv) |
                  ((in.off_x != 0.0f || in.off_y != 0.0f || in.off_z != 0.0f) ? kBatchOff : 0);
        b.quad_gx = ceil_div(in.W + 1, 32) * (in.H + 1);
        b.tiles_bwd = fp_tiles_per_view(in.U, in.V, b.tile_bwd);
        host[i] = b;
        item_fwd[i + 1] = item_fwd[i] + fp_tiles_per_view(in.U, in.V, b.tile_fwd) * in.A;
        item_bwd[i + 1] = item_bwd[i] + b.tiles_bwd * in.A;
        quad_block[i + 1] = quad_block[i] + (long long)b.quad_gx * ceil_div(in.D + 2, 32);
        view[i + 1] = view[i] + in.A;
        const long long voxels = (long long)in.D * in.H * in.W;
        fold_block[i + 1] = fold_block[i] + (in.grad_volume ? (voxels + kFoldChunk - 1) / kFoldChunk : 0);
        rays += (long long)in.A * in.U * in.V;
        if (!in.grad_projections || !in.grad_geometry) backward_ready = 0;
    }
    DGC_REQUIRE(quad_block[n] < (1LL << 31) && view[n] < (1LL << 31) && fold_block[n] < (1LL << 31),
                "batch exceeds the 2^31 block limit of one launch");

    cudaStream_t s = (cudaStream_t)stream;
    const BatchTables t = tables_at(workspace, n);
    // pageable sources: each copy returns once its data is staged, so the
    // host vectors may go out of scope afterwards
    DGC_CUDA(cudaMemcpyAsync(const_cast<BatchInstance*>(t.inst), host.data(),
                             sizeof(BatchInstance) * (size_t)n, cudaMemcpyHostToDevice, s));
    const long long* dst[5] = {t.item_fwd, t.item_bwd, t.quad_block, t.view, t.fold_block};
    for (int k = 0; k < 5; ++k)
        DGC_CUDA(cudaMemcpyAsync(const_cast<long long*>(dst[k]), prefix.data() + (size_t)k * (n + 1),
                                 sizeof(long long) * (size_t)(n + 1), cudaMemcpyHostToDevice, s));

    int gf = 0, gb = 0;
    int rc = batch_persistent_grid(false, &gf);
    if (rc != DGC_OK) return rc;
    rc = batch_persistent_grid(true, &gb);
    if (rc != DGC_OK) return rc;
    memset(plan, 0, sizeof(*plan));
    plan->workspace = workspace;
    plan->n = n;
    plan->grid_forward = (int)std::min<long long>(gf, item_fwd[n]);
    plan->grid_backward = (int)std::min<long long>(gb, item_bwd[n]);
    plan->has_grad_volume = gpad_total > 0;
    plan->backward_ready = backward_ready;
    plan->items_forward = item_fwd[n];
    plan->items_backward = item_bwd[n];
    plan->quad_blocks = quad_block[n];
    plan->views = view[n];
    plan->fold_blocks = fold_block[n];
    plan->rays = rays;
    plan->grad_pad_offset = gpad_off;
    plan->grad_pad_bytes = gpad_total;
    plan->tables_bytes = tb;
    return DGC_OK;
}

static int check_plan(const dgc_batch_plan* plan) {
    DGC_REQUIRE(plan && plan->workspace && plan->n > 0, "plan was not prepared");
    return DGC_OK;
}

int dgc_batch_project(const dgc_batch_plan* plan, void* stream) {
    clear_error();
    int rc = check_plan(plan);
    if (rc != DGC_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const BatchTables t = tables_at(plan->workspace, plan->n);
    rc = batch_launch_quads(t, plan->quad_blocks, s);
    if (rc != DGC_OK) return rc;
    return batch_launch_forward(t, plan->grid_forward, s);
}

int dgc_batch_project_backward(const dgc_batch_plan* plan, int rebuild_quads, void* stream) {
    clear_error();
    int rc = check_plan(plan);
    if (rc != DGC_OK) return rc;
    DGC_REQUIRE(plan->backward_ready,
                "every instance of the batch needs grad_projections and grad_geometry");
    cudaStream_t s = (cudaStream_t)stream;
    const BatchTables t = tables_at(plan->workspace, plan->n);
    if (rebuild_quads) {
        rc = batch_launch_quads(t, plan->quad_blocks, s);
        if (rc != DGC_OK) return rc;
    }
    if (plan->grad_pad_bytes)
        DGC_CUDA(cudaMemsetAsync(static_cast<char*>(plan->workspace) + plan->grad_pad_offset, 0,
                                 plan->grad_pad_bytes, s));
    return batch_launch_backward(t, plan->grid_backward, plan->views, plan->fold_blocks, s);
}

}  // extern "C"
