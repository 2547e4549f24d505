// fdk.cuh -- launch interface of the FDK filter.
#pragma once

#include <vector>

#include "common.cuh"

namespace dgc {

struct FdkArgs {
    const float* projections;  // [A][U][V]
    const float* sod;          // [A]
    const float* sid;          // [A]
    const float* taps;         // [U] filter taps h[0..U-1]
    float* filtered;           // [A][U][V]
    int A, U, V;
    float pixel_size;
    const float* uweight;      // [A][U] extra per-column weight (short-scan), or null
    // adjoint (fdk_launch_filter_adjoint): upstream gradient of `filtered`, the
    // forward output, the projection gradient (or null) and FP64 per-(view,
    // tile) partial sums (or null: no distance gradients)
    const float* grad_filtered;  // [A][U][V]
    const float* forward_out;    // [A][U][V]
    float* grad_projections;     // [A][U][V]
    double* partials;            // [A][tiles][2]
};

int fdk_taps_host(int U, double px, double alpha, std::vector<double>& out);
int fdk_upload_taps(int U, float px, float alpha, float* dst, cudaStream_t s);
int fdk_launch_filter(const FdkArgs& p, cudaStream_t s);
// Adjoint of the filter: grad_projections = c w H(g) and the per-view sums of
// g*y and H(g)*P*dw/dsid (partials), then dgc's distance gradients from them.
long long fdk_filter_tiles(int U, int V);
int fdk_launch_filter_adjoint(const FdkArgs& p, cudaStream_t s);
int fdk_reduce_distance_grads(const double* partials, int A, long long tiles, const float* sod,
                              const float* sid, float pixel_size, float* grad_sod,
                              float* grad_sid, cudaStream_t s);
// Parker short-scan weights w[a][u] of a scan over angles[0] .. angles[A-1].
int fdk_parker_weights(const float* angles, const float* sid, int A, int U, float pixel_size,
                       float* weights, cudaStream_t s);

}  // namespace dgc
