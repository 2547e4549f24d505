// backprojector.cuh -- launch interface of the backprojector kernels.
#pragma once

#include "common.cuh"

namespace dgc {

// Most warps (columns) in one CTA of the backprojection; most tile rules.
constexpr int kBpMaxWarps = 16;
constexpr int kBpMaxTileRules = 16;

// Per-view terms shared by every voxel of a view (48 bytes).
struct ViewRow {
    float c, s;          // cos, sin of the view angle
    float ds_u, ds_n;    // source offset in the rotating detector frame
    float ds_v;          // src_z
    float sod, sid, u0, v0;
    float pad0, pad1, pad2;
};

struct BpArgs {
    const ViewRow* vt;     // [A]
    const float4* pquads;  // [A][U-1][V-1]
    int A, U, V, D, H, W;
    float pixel_size, inv_pixel, voxel_size;
    float off_x, off_y, off_z;
    // forward
    float* volume;     // [D][H][W]
    int cta_x, cta_y;  // forward: columns per CTA along x and y (cta_x*cta_y <= kBpMaxWarps)
    int kz_backward;   // backward: Z blocking chosen with the partials' size (0: choose)
    float out_scale;   // FDK epilogue scale (pi/A)
    int clamp;         // FDK epilogue: clamp at 0 (0 for a view-sharded partial volume)
    // backward
    const float* grad_volume;  // [D][H][W]
    float* grad_projections;   // [A][U][V], zeroed by the caller; null: not computed
    double* partials;          // [A][8][blocks]
};

int bp_view_table(const Geometry& g, int A, ViewRow* vt, cudaStream_t s);
int build_proj_quads(const float* P, int A, int U, int V, float4* PQ, cudaStream_t s);
int bp_launch_forward(const BpArgs& p, bool fdk, cudaStream_t s);
int bp_launch_backward(const BpArgs& p, cudaStream_t s);
int bp_clamp_volume(float* volume, long long n, cudaStream_t s);
long long bp_backward_blocks(int D, int H, int W, int kz);
// Tiles of a call with volume depth D and A views (rules, overrides, built-in
// choice) and the rule table behind dgc_bp_add_tile_rule (0 ok, -1 invalid,
// -2 table full).
int bp_kz_forward(int D, int A);
int bp_kz_backward(int D, int A);
void bp_forward_cta(int D, int A, int& cx, int& cy);
int bp_add_tile_rule(int d_max, int a_max, int kz_forward, int kz_backward, int cta_x, int cta_y);
void bp_clear_tile_rules();
int bp_reduce_partials(const double* partials, int A, long long nblocks, const GeometryGrad& out,
                       cudaStream_t s);

}  // namespace dgc
