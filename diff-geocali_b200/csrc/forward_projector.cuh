// forward_projector.cuh -- launch interface of the forward projector kernels.
#pragma once

#include "common.cuh"

namespace dgc {

struct FpArgs {
    Geometry g;
    int D, H, W, A, U, V;
    float pixel_size, step_size, voxel_size, inv_voxel;
    float off_x, off_y, off_z;
    // edge-replicated, z-fastest quad-packed volume Q[(yp*(W+1) + xp)*(D+2) + zp]
    const float4* quads;
    uint32_t zq_x, zq_y, zq_bias;
    // forward output [A][U][V]
    float* projections;
    // backward
    const float* grad_projections;  // [A][U][V]
    float* grad_pad;                // level records R[(yp*(W+1) + xp)*(D+2) + zp][4] or null
    uint32_t gz_x, gz_y, gz_bias;
    double* partials;  // [A][tiles][8]
    int* error;        // device word set to 1 when a bounded wait gives up (TMA arm), or null
    int view_block;    // CTA order: 0 = u tile fastest; B > 0 = views in blocks of B (tile_coord),
                       // and the L1 forward's warps as 4 x 8 ray patches (tile_ray)
};

// Ray tile of a CTA: TU detector columns x (256/TU) rows; the 32 lanes of a
// warp run along V (wu = 1).
struct FpTile {
    int tu;
    int wu;
};

// One instance of a batched launch (an entry of the device-resident table).
enum : int { kBatchDiv = 1, kBatchOff = 2 };
constexpr int kFoldChunk = 2048;

struct BatchInstance {
    FpArgs p;              // arguments with this instance's quads, outputs and workspace slices
    const float* volume;   // [D][H][W]
    float* grad_volume;    // [D][H][W]; null: no volume gradient
    GeometryGrad gout;     // eight [A] outputs
    int tile_fwd, tile_bwd;  // columns per CTA tile (forward 8/4/2, backward 8/4)
    int flags;             // kBatchDiv (non power-of-two voxel) | kBatchOff (non-zero ROI
                           // offset)
    int quad_gx;           // blocks along x of the quads build
    long long tiles_bwd;   // backward tiles per view
};

// Device pointers of a prepared batch; the prefix arrays have n+1 entries.
struct BatchTables {
    const BatchInstance* inst;
    int n;
    const long long* item_fwd;     // forward work items
    const long long* item_bwd;     // backward work items
    const long long* quad_block;   // quads-build blocks
    const long long* view;         // views
    const long long* fold_block;   // gradient-fold blocks
    unsigned long long* counters;  // [0] forward queue, [1] backward queue
};

int batch_launch_quads(const BatchTables& t, long long blocks, cudaStream_t s);
int batch_launch_forward(const BatchTables& t, int grid, cudaStream_t s);
int batch_launch_backward(const BatchTables& t, int grid, long long views, long long fold_blocks,
                          cudaStream_t s);
int batch_persistent_grid(bool backward, int* grid);

// Argument checks of dgc_project (messages as the reference's host wrapper).
int fp_check_args(int D, int H, int W, int A, int U, int V, float pixel_size, float step_size,
                  float voxel_size, const Geometry& g);

void fp_fill_layout(FpArgs& p);
long long fp_tiles_per_view(int U, int V, int tu);
// Volume gradient of the backward: the weights of a lane's consecutive
// samples in one cell are added in registers and emitted as 16-byte vector
// reductions into a cell-major buffer of level records (4 floats per cell,
// fp_record_buffer_floats), then folded onto the voxels (fp_fold_records).
size_t fp_record_buffer_floats(int D, int H, int W);
int fp_fold_records(const float* records, int D, int H, int W, float* grad, cudaStream_t s);
int build_volume_quads(const float* vol, int D, int H, int W, float4* quads, cudaStream_t s);
// The forward's arm, slab, unroll and CTA order for a volume (the arm rules).
struct FpArm {
    int arm = 0, slab = 0, unroll = 1, view_block = 0;
};
// With arm 2 (z pairs) p.quads must hold build_volume_pairs' layout, else the quads.
int fp_launch_forward(const FpArgs& p, const FpTile& tile, const FpArm& arm, cudaStream_t s);
int build_volume_pairs(const float* vol, int D, int H, int W, float2* pairs, cudaStream_t s);
// Forward arm per volume size: 0 = quads through L1 (fp_forward_kernel, march
// unrolled 1 or 2 times), 1 = bricks staged by TMA (fp_forward_tma_kernel,
// slab of 2 or 4 cells), 2 = z pairs through L1 (fp_forward_pairs_kernel,
// half the quads' bytes); and the CTA order (view_block, tile_coord); rules
// registered by the autotuner (0 ok, -1 invalid, -2 table full).
int fp_add_arm_rule(long long voxels_max, int arm, int slab, int unroll, int view_block);
void fp_clear_arm_rules();
void fp_forward_arm(int D, int H, int W, int* arm, int* slab, int* unroll, int* view_block);
FpArm fp_forward_arm(int D, int H, int W);
int fp_launch_backward(const FpArgs& p, const FpTile& tile, bool gradvol, cudaStream_t s);
int fp_launch_counts(const FpArgs& p, int64_t* counts, cudaStream_t s);
// Fused projection -> masked squared error -> geometry-gradient terms (8-column
// tiles); p.partials [A][tiles][8], loss_partials [A][tiles].
// Columns per CTA tile of the fused calibration step (by volume size).
int fp_mse_tile(int D, int H, int W);
// tile: columns per CTA (fp_mse_tile(), decided with the partials' size)
int fp_launch_mse_grad(const FpArgs& p, int tile, const float* measured, const float* mask,
                       float scale, double* loss_partials, cudaStream_t s);
int fp_sum_partials(const double* x, long long n, double scale, double* out, cudaStream_t s);
int fp_reduce_partials(const double* partials, int A, long long tiles, const GeometryGrad& out,
                       cudaStream_t s);

}  // namespace dgc
