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
    float* grad_pad;                // G[(yp*(W+2) + xp)*(D+2) + zp] or null
    uint32_t gz_x, gz_y, gz_bias;
    double* partials;  // [A][tiles][8]
};

// Ray tile of a CTA: TU detector columns x (256/TU) rows; the 32 lanes of a
// warp run along V (wu = 1).
struct FpTile {
    int tu;
    int wu;
};

void fp_fill_layout(FpArgs& p);
long long fp_tiles_per_view(int U, int V, int tu);
int build_volume_quads(const float* vol, int D, int H, int W, float4* quads, cudaStream_t s);
int fp_launch_forward(const FpArgs& p, const FpTile& tile, cudaStream_t s);
int fp_launch_backward(const FpArgs& p, const FpTile& tile, bool gradvol, cudaStream_t s);
int fp_launch_counts(const FpArgs& p, int64_t* counts, cudaStream_t s);
int fp_reduce_partials(const double* partials, int A, long long tiles, const GeometryGrad& out,
                       cudaStream_t s);
int fp_fold_gradient(const float* gpad, int D, int H, int W, float* grad, cudaStream_t s);

}  // namespace dgc
