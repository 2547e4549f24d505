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
    const float* uweight = nullptr;  // [A][U] extra per-column weight (short-scan), or null
    // adjoint (fdk_launch_filter_adjoint): upstream gradient of `filtered`, the
    // forward output, the projection gradient (or null) and FP64 per-(view,
    // tile) partial sums (or null: no distance gradients)
    const float* grad_filtered = nullptr;  // [A][U][V]
    const float* forward_out = nullptr;    // [A][U][V]
    float* grad_projections = nullptr;     // [A][U][V]
    double* partials = nullptr;            // [A][tiles][kFdkPartials]
    // Preweight frame per view, each null for the reference's centred weight:
    // the source's distance to the detector plane (null: sid) and the pixel
    // indices (u, v) of the foot of the perpendicular from the source (null:
    // (U-1)/2, (V-1)/2).  The preweight is dist_n / |source - pixel|, the
    // cosine of the ray's angle to the detector normal.
    const float* frame_dist = nullptr;  // [A]
    const float* frame_u = nullptr;     // [A]
    const float* frame_v = nullptr;     // [A]
    int frame_grads = 0;  // adjoint: also the sums for the frame-centre gradients
};

// FP64 sums per (view, tile) of the adjoint: g*y, H(g) P dw/ddist,
// H(g) P u_c/|r|^3, H(g) P v_c/|r|^3 (u_c, v_c in length units).
constexpr int kFdkPartials = 4;

int fdk_taps_host(int U, double px, double alpha, std::vector<double>& out);
int fdk_upload_taps(int U, float px, float alpha, float* dst, cudaStream_t s);
int fdk_launch_filter(const FdkArgs& p, cudaStream_t s);
// Adjoint of the filter: grad_projections = c w H(g) and the per-view sums of
// g*y and H(g)*P*dw/dsid (partials), then dgc's distance gradients from them.
long long fdk_filter_tiles(int U, int V);
int fdk_launch_filter_adjoint(const FdkArgs& p, cudaStream_t s);
// Per-view gradients from the partials: sod, sid, and, where the frame was
// given, its distance and centres (any output may be null).
struct FdkGrads {
    float* sod;
    float* sid;
    float* frame_dist;
    float* frame_u;
    float* frame_v;
};
int fdk_reduce_distance_grads(const double* partials, int A, long long tiles, const FdkArgs& p,
                              const FdkGrads& g, cudaStream_t s);
// Parker short-scan weights w[a][u] of a scan over angles[0] .. angles[A-1];
// the fan angle of column u is atan((u - centre) * pixel / dist) with the
// frame's centre and distance (null: (U-1)/2 and sid).
int fdk_parker_weights(const float* angles, const float* sid, const float* frame_dist,
                       const float* frame_u, int A, int U, float pixel_size, float* weights,
                       cudaStream_t s);

}  // namespace dgc
