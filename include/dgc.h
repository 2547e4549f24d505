/*
 * dgc.h -- C ABI of libdgc, the sm_100a cone-beam CT operators.
 *
 * Every entry point takes plain device pointers, sizes and scalars, returns a
 * status code (DGC_OK == 0) and launches asynchronously on the CUDA stream
 * passed as `stream` (a cudaStream_t; NULL selects the legacy default stream).
 * On failure, dgc_last_error() returns a message for the calling thread.
 *
 * Memory: all inputs and outputs are caller-owned device buffers, C-contiguous
 * float32.  Outputs are fully overwritten.  Kernels that need scratch memory
 * take a caller-owned device `workspace` of at least the size reported by the
 * matching *_workspace_bytes() query (256-byte aligned); no entry point
 * allocates device memory.
 *
 * Geometry: eight per-view float32 arrays of length A, in the reference's
 * order: angles [rad], sid (source-detector distance), sod (source-origin
 * distance), det_u0, det_v0 (detector centre indices, pixels), src_x, src_y,
 * src_z (world source offsets).  Volumes are [D,H,W] (W fastest), projections
 * [A,U,V] (V fastest).  Voxel (z,y,x) sits at ((x-W/2)*voxel+off_x,
 * (y-H/2)*voxel+off_y, (z-D/2)*voxel+off_z).
 *
 * Each entry point names the reference interface it replaces (paths within
 * the TomSHINING/diff-geoCali project).
 */
#ifndef DGC_H
#define DGC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGC_ABI_VERSION 1

enum dgc_status {
    DGC_OK = 0,
    DGC_ERR_INVALID_ARGUMENT = 1, /* the reference raises RuntimeError (TORCH_CHECK) */
    DGC_ERR_CUDA = 2,             /* a CUDA runtime call or launch failed */
    DGC_ERR_WORKSPACE = 3,        /* workspace missing, misaligned or too small */
    DGC_ERR_UNSUPPORTED = 4       /* sizes beyond the library's index limits */
};

/* ABI version of the loaded library (DGC_ABI_VERSION). */
int dgc_abi_version(void);

/* Message of the last failure on the calling thread ("" if none). */
const char* dgc_last_error(void);

/* ---------------------------------------------------------------------- */
/* Forward projector: p[a,u,v] = step * sum_k trilinear(volume, O + t_k d) */
/* ---------------------------------------------------------------------- */

/* Scratch of dgc_project / dgc_project_sample_counts (edge-replicated
 * quad-packed copy of the volume). */
size_t dgc_project_workspace_bytes(int D, int H, int W, int A, int U, int V);

/* Replaces src_cbct_forwardprojector_cuda.forward
 * (csrc/src_cbct_forwardprojector_cuda.cu:566-631, kernel 258-339). */
int dgc_project(const float* volume, int D, int H, int W,
                const float* angles, const float* sid, const float* sod,
                const float* det_u0, const float* det_v0,
                const float* src_x, const float* src_y, const float* src_z, int A,
                float pixel_size, int U, int V, float step_size, float voxel_size,
                float off_x, float off_y, float off_z,
                float* projections,
                void* workspace, size_t workspace_bytes, void* stream);

/* Number of trilinear samples of every ray under the kernel's FP32 stepping
 * rule (counts[a,u,v], int64); the algorithmic-work figure of a projection.
 * No counterpart in the reference (measurement support). */
int dgc_project_sample_counts(int D, int H, int W,
                              const float* angles, const float* sid, const float* sod,
                              const float* det_u0, const float* det_v0,
                              const float* src_x, const float* src_y, const float* src_z,
                              int A, float pixel_size, int U, int V, float step_size,
                              float voxel_size, float off_x, float off_y, float off_z,
                              int64_t* counts, void* stream);

/* Scratch of dgc_project_backward. */
size_t dgc_project_backward_workspace_bytes(int D, int H, int W, int A, int U, int V,
                                            int compute_grad_volume);

/* Replaces src_cbct_forwardprojector_cuda.backward
 * (csrc/src_cbct_forwardprojector_cuda.cu:634-729, kernel 342-528).
 * grad_volume [D,H,W] may be NULL when compute_grad_volume == 0.  The eight
 * geometry gradients [A] are reduced per view in FP64 in a fixed order
 * (bitwise reproducible); the volume gradient uses float atomics. */
int dgc_project_backward(const float* grad_projection, const float* volume,
                         int D, int H, int W,
                         const float* angles, const float* sid, const float* sod,
                         const float* det_u0, const float* det_v0,
                         const float* src_x, const float* src_y, const float* src_z, int A,
                         float pixel_size, int U, int V, float step_size, float voxel_size,
                         int compute_grad_volume, float off_x, float off_y, float off_z,
                         float* grad_volume, float* grad_angles, float* grad_sid,
                         float* grad_sod, float* grad_det_u0, float* grad_det_v0,
                         float* grad_src_x, float* grad_src_y, float* grad_src_z,
                         void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------- */
/* Voxel-driven FDK-weighted backprojector                                  */
/* ---------------------------------------------------------------------- */

/* Scratch of dgc_backproject (per-view table + quad-packed projections). */
size_t dgc_backproject_workspace_bytes(int A, int U, int V, int D, int H, int W);

/* Replaces src_cbct_backprojector_cuda.forward
 * (csrc/src_cbct_backprojector_cuda.cu:344-420, kernel 15-98). */
int dgc_backproject(const float* projections, int A, int U, int V,
                    const float* angles, const float* sid, const float* sod,
                    const float* det_u0, const float* det_v0,
                    const float* src_x, const float* src_y, const float* src_z,
                    float pixel_size, int D, int H, int W, float voxel_size,
                    float off_x, float off_y, float off_z,
                    float* volume,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Scratch of dgc_backproject_backward. */
size_t dgc_backproject_backward_workspace_bytes(int A, int U, int V, int D, int H, int W);

/* Replaces src_cbct_backprojector_cuda.backward
 * (csrc/src_cbct_backprojector_cuda.cu:423-522, kernel 101-295).
 * Writes grad_projections [A,U,V] and the eight geometry gradients [A]
 * (per-view FP64 reductions in a fixed order).  grad_projections may be NULL:
 * the projection gradient (the bilinear scatter) is then skipped, which the
 * reference always computes. */
int dgc_backproject_backward(const float* grad_volume, const float* projections,
                             int A, int U, int V,
                             const float* angles, const float* sid, const float* sod,
                             const float* det_u0, const float* det_v0,
                             const float* src_x, const float* src_y, const float* src_z,
                             float pixel_size, int D, int H, int W, float voxel_size,
                             float off_x, float off_y, float off_z,
                             float* grad_projections, float* grad_angles, float* grad_sid,
                             float* grad_sod, float* grad_det_u0, float* grad_det_v0,
                             float* grad_src_x, float* grad_src_y, float* grad_src_z,
                             void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------- */
/* FDK                                                                      */
/* ---------------------------------------------------------------------- */

/* Host-only: the U filter taps h[0..U-1] of the zero-padded Ram-Lak x Hann
 * filter (filtering.py:87-103) as a symmetric Toeplitz kernel, FP64. */
int dgc_fdk_filter_taps(int U, double pixel_size, double alpha, double* taps);

/* Scratch of dgc_fdk_filter. */
size_t dgc_fdk_filter_workspace_bytes(int A, int U, int V);

/* Replaces cbct_backprojector.filtering.fdk_filter (filtering.py:54-104):
 * centred cosine preweight, ramp x Hann filter along U, pixel*sid/sod scale.
 * sod and sid are per-view device arrays [A]. */
int dgc_fdk_filter(const float* projections, int A, int U, int V, float pixel_size,
                   const float* sod, const float* sid, float alpha,
                   float* filtered,
                   void* workspace, size_t workspace_bytes, void* stream);

/* dgc_fdk_filter with the cosine preweight taken in a per-view frame: w =
 * dist_n / sqrt(dist_n^2 + ((u - fu) px)^2 + ((v - fv) px)^2), the cosine of
 * the ray's angle to the detector normal for a source at distance dist_n =
 * frame_dist[a] from the detector plane whose perpendicular meets it at pixel
 * (fu, fv) = (frame_u[a], frame_v[a]).  Each of frame_dist, frame_u, frame_v
 * is a device array [A] or NULL for the reference's centred weight (sid,
 * (U-1)/2, (V-1)/2); with all three NULL this is dgc_fdk_filter, bit for bit.
 * frame_dist must be positive (not checked on the device).  The reference's
 * preweight is centred whatever the detector and source offsets
 * (filtering.py:1-8, 70-71, 82-85; README.md:115); no counterpart there.  Same
 * workspace as dgc_fdk_filter. */
int dgc_fdk_filter_ex(const float* projections, int A, int U, int V, float pixel_size,
                      const float* sod, const float* sid, const float* frame_dist,
                      const float* frame_u, const float* frame_v, float alpha, float* filtered,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Maximum detector width U accepted by dgc_fdk_filter_noalloc. */
#define DGC_FDK_NOALLOC_MAX_U 8192

/* No counterpart in the reference.  dgc_fdk_filter for callers that cannot
 * allocate device memory: a host application that owns the GPU's memory and
 * hands each library a fixed budget, a plugin that must not grow the process's
 * device footprint, or a latency-bound pipeline that keeps cudaMalloc and
 * cudaFree (which can synchronise the device) out of its steady state.  It
 * takes no workspace and allocates nothing: its scratch, the filter's spectrum
 * and taps, lives in one static device array of 98 KiB
 * (DGC_FDK_NOALLOC_MAX_U + 1 doubles and DGC_FDK_NOALLOC_MAX_U floats) that
 * every GPU loading the library holds until the process exits; U above
 * DGC_FDK_NOALLOC_MAX_U returns DGC_ERR_UNSUPPORTED.  Two small kernels write
 * the taps on the device, in stream order before the filter, so a call reads
 * no host memory after it returns and never waits on the host for earlier
 * work in its stream.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and keeps it for the process; make that
 * first call before any stream capture.  A cudaDeviceReset of that device
 * invalidates the kept address, so do not call this entry point on a device
 * after resetting it.  Every call rewrites the spectrum and taps[0..U-1]
 * before its filter reads them, so nothing needs to start at zero, but all
 * calls share the one array: calls that overlap on the GPU (different
 * streams, no ordering between them) race on it.  Same inputs and outputs as
 * dgc_fdk_filter; results equal its within the taps' FP64 rounding. */
int dgc_fdk_filter_noalloc(const float* projections, int A, int U, int V, float pixel_size,
                           const float* sod, const float* sid, float alpha,
                           float* filtered, void* stream);

/* Scratch of dgc_fdk_filter_backward. */
size_t dgc_fdk_filter_backward_workspace_bytes(int A, int U, int V);

/* Gradients of dgc_fdk_filter, which the reference's torch implementation of
 * fdk_filter (filtering.py:54-104) gets from autograd: for the upstream
 * gradient grad_filtered of filtered = c H(w P) (H the symmetric Toeplitz
 * filter along U, w = sid/dist the centred cosine weight, c = pixel*sid/sod),
 *   grad_projections = c w H(grad_filtered)                       [A,U,V]
 *   grad_sid[a] = sum(g y)/sid + c sum(H(g) P dw/dsid),  grad_sod[a] = -sum(g y)/sod
 * with y = filtered (the forward's output) and dw/dsid = (u^2+v^2)/dist^3; the
 * per-view sums in FP64, fixed order.  Any of grad_projections, grad_sod,
 * grad_sid may be NULL (not computed); projections and filtered are read only
 * for the distance gradients. */
int dgc_fdk_filter_backward(const float* grad_filtered, const float* projections,
                            const float* filtered, int A, int U, int V, float pixel_size,
                            const float* sod, const float* sid, float alpha,
                            float* grad_projections, float* grad_sod, float* grad_sid,
                            void* workspace, size_t workspace_bytes, void* stream);

/* Gradients of dgc_fdk_filter_ex: those of dgc_fdk_filter_backward (with the
 * frame's dist_n in place of sid inside the preweight; grad_sid then holds
 * only sum(g y)/sid, the scale's share) and, for each frame array given, its
 * per-view gradient: grad_frame_dist = c sum(H(g) P dw/ddist_n),
 * grad_frame_u = c dist_n px sum(H(g) P (u - fu) px / r^3) and grad_frame_v
 * likewise, r the source-pixel distance.  A frame gradient needs its frame
 * array; any gradient may be NULL.  Same workspace as
 * dgc_fdk_filter_backward.  No counterpart in the reference. */
int dgc_fdk_filter_backward_ex(const float* grad_filtered, const float* projections,
                               const float* filtered, int A, int U, int V, float pixel_size,
                               const float* sod, const float* sid, const float* frame_dist,
                               const float* frame_u, const float* frame_v, float alpha,
                               float* grad_projections, float* grad_sod, float* grad_sid,
                               float* grad_frame_dist, float* grad_frame_u, float* grad_frame_v,
                               void* workspace, size_t workspace_bytes, void* stream);

/* Scratch of dgc_reconstruct_fdk. */
size_t dgc_reconstruct_fdk_workspace_bytes(int A, int U, int V, int D, int H, int W);

/* Replaces cbct_backprojector.filtering.reconstruct_fdk (filtering.py:107-198):
 * filter, backproject all views, * pi/A, clamp at 0 -- one filter launch and
 * one backprojection launch over all views. */
int dgc_reconstruct_fdk(const float* projections, int A, int U, int V,
                        const float* angles, const float* sid, const float* sod,
                        const float* det_u0, const float* det_v0,
                        const float* src_x, const float* src_y, const float* src_z,
                        float pixel_size, int D, int H, int W, float voxel_size,
                        float off_x, float off_y, float off_z, float alpha,
                        float* volume,
                        void* workspace, size_t workspace_bytes, void* stream);

/* Parker short-scan weights w[a][u] (Parker, Med. Phys. 9(2), 1982) of a scan
 * over angles[0] .. angles[A-1] (monotone, range pi + 2*Gamma with Gamma at
 * least the largest fan angle atan(((U-1)/2 * pixel_size) / sid)): each ray
 * and its conjugate weigh 1 together.  The reference's FDK assumes a full
 * circle (README.md:115, filtering.py:1-8); no counterpart there. */
int dgc_parker_weights(const float* angles, const float* sid, int A, int U, float pixel_size,
                       float* weights, void* stream);

/* dgc_parker_weights with the fan angle of column u taken in the preweight
 * frame of dgc_fdk_filter_ex: gamma = atan((u - frame_u[a]) px /
 * frame_dist[a]) (either array NULL: (U-1)/2, sid).  No counterpart in the
 * reference. */
int dgc_parker_weights_ex(const float* angles, const float* sid, const float* frame_dist,
                          const float* frame_u, int A, int U, float pixel_size, float* weights,
                          void* stream);

/* dgc_reconstruct_fdk with a per-(view, column) weight multiplied into the
 * cosine preweight (uweights [A][U], e.g. dgc_parker_weights; NULL for none)
 * and the angular factor angle_scale in place of pi/A (the view spacing for
 * a Parker-weighted short scan).  Same workspace as dgc_reconstruct_fdk.
 * Extends filtering.py:107-198 to short scans; no counterpart in the
 * reference. */
int dgc_reconstruct_fdk_weighted(const float* projections, int A, int U, int V,
                                 const float* angles, const float* sid, const float* sod,
                                 const float* det_u0, const float* det_v0,
                                 const float* src_x, const float* src_y, const float* src_z,
                                 float pixel_size, int D, int H, int W, float voxel_size,
                                 float off_x, float off_y, float off_z, float alpha,
                                 const float* uweights, float angle_scale, float* volume,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* One rank's share of a view-sharded FDK reconstruction: dgc_reconstruct_fdk_weighted
 * over this rank's views without the final clamp, so that the partial volumes
 * of all ranks can be summed (an all-reduce) before dgc_clamp_volume.
 * angle_scale is pi / (views over all ranks) for a full scan.  Same workspace
 * as dgc_reconstruct_fdk.  The reference reconstructs on one device
 * (filtering.py:107-198); no counterpart there. */
int dgc_reconstruct_fdk_partial(const float* projections, int A, int U, int V,
                                const float* angles, const float* sid, const float* sod,
                                const float* det_u0, const float* det_v0,
                                const float* src_x, const float* src_y, const float* src_z,
                                float pixel_size, int D, int H, int W, float voxel_size,
                                float off_x, float off_y, float off_z, float alpha,
                                const float* uweights, float angle_scale, float* volume,
                                void* workspace, size_t workspace_bytes, void* stream);

/* The general FDK reconstruction the three above specialise: the filter in
 * the preweight frame of dgc_fdk_filter_ex (frame_dist, frame_u, frame_v,
 * each NULL for the centred default), the per-(view, column) weights
 * uweights (NULL for none), the angular factor angle_scale, then the clamp at
 * zero if clamp != 0.  Same workspace as dgc_reconstruct_fdk.  Extends
 * filtering.py:107-198; no counterpart in the reference. */
int dgc_reconstruct_fdk_ex(const float* projections, int A, int U, int V,
                           const float* angles, const float* sid, const float* sod,
                           const float* det_u0, const float* det_v0,
                           const float* src_x, const float* src_y, const float* src_z,
                           float pixel_size, int D, int H, int W, float voxel_size,
                           float off_x, float off_y, float off_z, float alpha,
                           const float* frame_dist, const float* frame_u, const float* frame_v,
                           const float* uweights, float angle_scale, int clamp, float* volume,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Backprojector tile rules (what the autotuner chose per shape bucket): a
 * call with volume depth D <= d_max and A <= a_max views uses Z blocking
 * kz_forward / kz_backward (32*kz voxels of a column per warp; 1, 2, 4 or 8,
 * 0 = built-in choice) and a cta_x x cta_y patch of columns per CTA in the
 * forward (both 0 = built-in 8 x 1; cta_x*cta_y <= 16).  Rules are tried in
 * the order they were added (at most 16).  Results do not depend on the tiles
 * beyond float-summation order (the forward's not at all).  No counterpart in
 * the reference. */
int dgc_bp_add_tile_rule(int d_max, int a_max, int kz_forward, int kz_backward, int cta_x,
                         int cta_y);
int dgc_bp_clear_tile_rules(void);
/* The tiles a call with depth D and A views uses. */
int dgc_bp_tiles(int D, int A, int* kz_forward, int* kz_backward, int* cta_x, int* cta_y);

/* Forward-projector arm rules (what the autotuner chose per volume size): a
 * dgc_project of D*H*W <= voxels_max voxels runs arm 0 (quad loads through
 * L1, fp_forward_kernel, its march loop unrolled `unroll` = 1 or 2 times),
 * arm 1 (volume bricks staged in shared memory by TMA, slab_cells = 2 or 4
 * cells per slab along the bundle's main axis; unroll 1) or arm 2 (the
 * volume as z pairs, half the quads' bytes, four 8-byte loads per cell;
 * unroll 1), with its CTAs in
 * the order view_block: 0 = every u tile of a view, then the next view;
 * B > 0 = inside a detector band, views in blocks of B, the view fastest
 * inside a block, and arm 0's warps as patches of 4 detector columns x 8
 * rows instead of 32 rows of one column.  Rules are tried in the order they were added (at most
 * 16); without one, arm 0, unroll 1, and view blocks of 16 above 2^26 voxels
 * (order 0 below).  Every choice gives bitwise the same projections; the
 * fused calibration step (dgc_project_mse_grad) takes the same CTA order.
 * No counterpart in the reference. */
int dgc_fp_add_arm_rule(long long voxels_max, int arm, int slab_cells, int unroll,
                        int view_block);
int dgc_fp_clear_arm_rules(void);
/* The arm, slab, unroll and CTA order a dgc_project of a D x H x W volume uses. */
int dgc_fp_arm(int D, int H, int W, int* arm, int* slab_cells, int* unroll, int* view_block);

/* volume[i] = max(volume[i], 0) in place (NaN stays NaN): the clamp that ends
 * an FDK reconstruction (filtering.py:197), after the partial volumes of a
 * view-sharded reconstruction have been summed. */
int dgc_clamp_volume(float* volume, long long n, void* stream);

/* ---------------------------------------------------------------------- */
/* Tensor-core GEMM of the warm-start network (no counterpart in the        */
/* reference: its calibration pipeline is not shipped)                      */
/* ---------------------------------------------------------------------- */

/* C[m,n] = alpha * sum_k A[m,k] B[n,k] (+ bias[n]) (then ReLU if relu != 0),
 * on the tcgen05 tensor cores with fp32 accumulation in tensor memory.
 * A [M x K] and B [N x K] are row-major bf16 with 16-byte aligned rows
 * (lda, ldb multiples of 8, K a multiple of 8); C is bf16 (c_bf16 = 1) or
 * fp32, row stride ldc; accumulate = 1 adds into an fp32 C.  error_flag is a
 * device int set to 1 if a pipeline wait of the kernel timed out. */
int dgc_gemm_bf16(const void* A, const void* B, void* C, const float* bias, int M, int N, int K,
                  int lda, int ldb, int ldc, int c_bf16, int relu, int accumulate, float alpha,
                  int* error_flag, void* stream);

/* Scratch of dgc_project_mse_grad. */
size_t dgc_project_mse_grad_workspace_bytes(int D, int H, int W, int A, int U, int V);

/* One geometry-calibration step fused into one ray march: the projection p of
 * dgc_project, the loss  *loss = scale * sum(mask * (p - measured)^2)  (FP64,
 * fixed-order sums) and the eight geometry gradients of that loss (those of
 * dgc_project_backward with grad_projection = 2*scale*mask*(p - measured)),
 * without the volume gradient.  mask may be NULL (all ones); projections may
 * be NULL (not stored).  Replaces the reference's forward + backward pair
 * (csrc/src_cbct_forwardprojector_cuda.cu:566-729) for a masked MSE loss,
 * which the reference composes in Python; one march instead of two. */
int dgc_project_mse_grad(const float* volume, int D, int H, int W,
                         const float* angles, const float* sid, const float* sod,
                         const float* det_u0, const float* det_v0,
                         const float* src_x, const float* src_y, const float* src_z,
                         int A, float pixel_size, int U, int V, float step_size,
                         float voxel_size, float off_x, float off_y, float off_z,
                         const float* measured, const float* mask, float scale,
                         float* projections, double* loss,
                         float* grad_angles, float* grad_sid, float* grad_sod,
                         float* grad_det_u0, float* grad_det_v0,
                         float* grad_src_x, float* grad_src_y, float* grad_src_z,
                         void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------- */
/* Raw frames to line integrals                                             */
/* ---------------------------------------------------------------------- */

/* out[a,u,v] = -log(max((raw - dark) / (flat - dark), min_ratio)), the
 * dark/flat-field correction and negative log the reference requires
 * upstream of its operators (README.md:108), fused with the transpose of
 * frames stored [A,V,U] (layout_avu = 1; U fastest) into the operators'
 * [A,U,V] (docs/USAGE.md:247-251).  raw: [A,V,U] or [A,U,V]; dark, flat: one
 * frame in the same layout, or NULL for 0 and 1.  No counterpart in the
 * reference's code. */
int dgc_preprocess(const float* raw, const float* dark, const float* flat, int A, int U, int V,
                   int layout_avu, float min_ratio, float* out, void* stream);

/* ---------------------------------------------------------------------- */
/* Batched forward projection + backward over uneven instances             */
/* ---------------------------------------------------------------------- */

/* One projection problem of a batch: the arguments of dgc_project and
 * dgc_project_backward.  grad_projections may alias projections (the
 * gradient of 0.5*|p|^2).  grad_volume NULL: no volume gradient.
 * grad_geometry: [8][A] (angles, sid, sod, det_u0, det_v0, src_x, src_y,
 * src_z).  tile_forward in {0, 8, 4, 2}, tile_backward in {0, 8, 4}: detector
 * columns per 256-ray CTA tile (0 = 8), normally chosen by the autotuner. */
typedef struct dgc_fp_instance {
    const float* volume;
    int D, H, W;
    const float *angles, *sid, *sod, *det_u0, *det_v0, *src_x, *src_y, *src_z;
    int A;
    float pixel_size;
    int U, V;
    float step_size, voxel_size, off_x, off_y, off_z;
    float* projections;
    const float* grad_projections;
    float* grad_volume;
    float* grad_geometry;
    int tile_forward, tile_backward;
} dgc_fp_instance;

/* A prepared batch: host-side, caller-owned, copyable; it refers to the
 * device tables that dgc_batch_prepare wrote into the workspace. */
typedef struct dgc_batch_plan {
    void* workspace;
    int n;
    int grid_forward, grid_backward; /* persistent CTAs */
    int has_grad_volume;
    int backward_ready;              /* every instance has grad_projections and grad_geometry */
    long long items_forward, items_backward, quad_blocks, views, fold_blocks;
    long long rays;                  /* sum of A*U*V */
    size_t grad_pad_offset, grad_pad_bytes;
    size_t tables_bytes;
} dgc_batch_plan;

/* Workspace of a batch: device tables plus, per instance, the quad-packed
 * volume, the padded volume gradient (if requested) and the per-tile FP64
 * partial sums.  No counterpart in the reference (which runs one problem per
 * call). */
size_t dgc_batch_workspace_bytes(const dgc_fp_instance* instances, int n);

/* Validates every instance (the checks of dgc_project, with the instance
 * index in the message), lays out the workspace and copies the device
 * tables into it on `stream` from host memory.  Call it outside stream
 * capture; afterwards dgc_batch_project / dgc_batch_project_backward may be
 * captured into a CUDA graph and replayed while the instances' buffers stay
 * valid.  No counterpart in the reference. */
int dgc_batch_prepare(const dgc_fp_instance* instances, int n, void* workspace,
                      size_t workspace_bytes, dgc_batch_plan* plan, void* stream);

/* Forward projections of every instance: one launch builds all quad-packed
 * volumes, one persistent launch marches every ray of every instance from an
 * (instance, view, ray tile) work queue.  Results equal dgc_project's
 * bitwise.  No counterpart in the reference. */
int dgc_batch_project(const dgc_batch_plan* plan, void* stream);

/* Backward of every instance (dgc_project_backward's outputs: volume and
 * geometry gradients).  rebuild_quads = 0 reuses the quad-packed volumes of
 * the last dgc_batch_project on this plan (the volumes unchanged since).
 * No counterpart in the reference. */
int dgc_batch_project_backward(const dgc_batch_plan* plan, int rebuild_quads, void* stream);

/* im2col of an NHWC bf16 image batch x [B,H,W,C] for a kh x kw convolution
 * (stride, zero padding pad): col [B*Ho*Wo][Kp] with column (ky*kw+kx)*C + c,
 * zero beyond kh*kw*C.  No counterpart in the reference. */
int dgc_im2col_nhwc_bf16(const void* x, int B, int H, int W, int C, int kh, int kw, int stride,
                         int pad, void* col, int Kp, void* stream);

/* Adjoint of dgc_im2col_nhwc_bf16 in fp32: dx [B,H,W,C] = col2im(col).
 * No counterpart in the reference. */
int dgc_col2im_nhwc_f32(const float* col, int B, int H, int W, int C, int kh, int kw, int stride,
                        int pad, int Kp, float* dx, void* stream);

/* ---------------------------------------------------------------------- */
/* Kernel timing (no counterpart in the reference; measurement support)     */
/* ---------------------------------------------------------------------- */

/* Enable (1) / disable (0) CUDA-event timing of every kernel launch. */
void dgc_trace_enable(int on);
/* Number of launches recorded since the last dgc_trace_clear(). */
int dgc_trace_count(void);
/* Name and device duration [ms] of record `index` (waits for its stop event). */
int dgc_trace_get(int index, char* name, int name_len, float* ms);
/* Drop all records. */
void dgc_trace_clear(void);

/* ---------------------------------------------------------------------- */
/* Ceilings (no counterpart in the reference; measurement support)          */
/* ---------------------------------------------------------------------- */

/* Launches one pass of 16-byte loads on every SM (ctas_per_sm CTAs of 256
 * threads per SM, `iterations` loads per thread, a multiple of 8): lane l of
 * a warp load reads element floor(l * lane_stride16 / 16) of a 1 KiB group
 * (lane_stride16 = 16: 512 contiguous bytes; 27: lanes 1.69 elements apart,
 * the backprojector's spread), groups in a random order.  level 1: the
 * groups of a 32 KiB window of `buffer` (resident in every SM's L1); level 2:
 * of the largest power-of-two prefix of `buffer` (at least 16 MiB; made far
 * larger than an SM's L1 and smaller than L2, its loads are served by L2).
 * *bytes receives the bytes the launch loads (16 per lane and load), for a
 * rate over the caller's event timing.  `buffer` should be zeroed; `sink` is
 * a float that the kernel never writes for zeroed input. */
int dgc_ceiling_gather(const void* buffer, size_t buffer_bytes, int level, int iterations,
                       int ctas_per_sm, int lane_stride16, float* sink, double* bytes,
                       void* stream);

/* Launches independent FFMA chains on every SM (ctas_per_sm CTAs of 256
 * threads per SM, 128 FFMA per iteration and thread); *warp_instructions
 * receives the FFMA warp instructions of the launch. */
int dgc_ceiling_issue(int iterations, int ctas_per_sm, float* sink, double* warp_instructions,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DGC_H */
