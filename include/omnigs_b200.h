/* omnigs_b200 -- B200-native equirectangular (lonlat) differentiable Gaussian rasterizer, C ABI.
 *
 * This is the drop-in boundary for OmniGS's camera_type = 3 path.  Every entry point takes plain
 * device pointers, sizes and a CUDA stream; no torch types cross it.  The LibTorch layer in
 * omnigs_b200/csrc/torch re-exports the reference's unchanged C++ surface on top of it:
 *
 *   RasterizeGaussiansCUDA          (src/rasterize_points.cu:49-164, include/rasterize_points.h:29-50)
 *   RasterizeGaussiansBackwardCUDA  (src/rasterize_points.cu:166-285, include/rasterize_points.h:52-74)
 *   markVisible                     (src/rasterize_points.cu:287-319, include/rasterize_points.h:76-80)
 *
 * Array conventions are the reference's: means3D [P,3], scales [P,3] (activated), rotations [P,4]
 * (r, x, y, z; used as given, not normalised), opacities [P] (activated), shs [P,M,3]
 * (coefficient-major, RGB inner), viewmatrix [16] = Tcw stored column-major (the row-major
 * storage of world_view_transform = Tcw^T), campos [3], background [3], images [3,H,W].
 * Optional inputs are NULL, as the reference's empty tensors are.
 *
 * The three state buffers (geometry, binning, image) are caller-owned device memory whose sizes
 * come from the *_bytes queries; their layout is private to this library.  They (and the batch
 * state buffer) must start on a 16-byte boundary, as cudaMalloc and the PyTorch allocator give
 * (OMNIGS_ERR_INVALID_ARGUMENT otherwise).  Nothing here allocates
 * device memory and nothing synchronises the host except omnigs_lonlat_read_status and
 * omnigs_lonlat_forward_early_status.  The instance count (num_rendered) is produced and consumed
 * on the device; the binning buffer is sized for a caller-chosen capacity and a pass that would
 * exceed it does no binning work and reports OMNIGS_STATUS_CAPACITY through the status word.
 *
 * Return codes: 0 on success, otherwise one of OMNIGS_ERR_*; omnigs_last_error() gives a message
 * (thread-local).  Kernels never trap: device-side failures are bits of the status word.
 */
#ifndef OMNIGS_B200_H_
#define OMNIGS_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* omnigs_stream_t; /* same type as cudaStream_t */

#define OMNIGS_OK 0
#define OMNIGS_ERR_INVALID_ARGUMENT 1
#define OMNIGS_ERR_BUFFER_TOO_SMALL 2
#define OMNIGS_ERR_CUDA 3
#define OMNIGS_ERR_UNSUPPORTED 4
#define OMNIGS_ERR_CAPACITY 5 /* num_rendered exceeds the binning capacity */
#define OMNIGS_ERR_DEVICE 6   /* a device-side status bit other than capacity is set */

/* Bits of the device status word (omnigs_lonlat_read_status). */
#define OMNIGS_STATUS_CAPACITY 1u /* num_rendered > binning capacity: binning and blend skipped */
#define OMNIGS_STATUS_LOOKBACK 2u /* a bounded cross-block wait gave up; results are invalid */
#define OMNIGS_STATUS_OVERFLOW 4u /* more than 2^30 - 1 instances */

#define OMNIGS_CAMERA_PINHOLE 1
#define OMNIGS_CAMERA_LONLAT 3

/* Bits of the forward/backward `flags` field.
 * OMNIGS_FLAG_RECOMPUTE_T: transmittance checkpointing.  The forward keeps no per-pixel state (the
 * image buffer, omnigs_lonlat_image_bytes_flags(W, H, OMNIGS_FLAG_RECOMPUTE_T), holds only the tile
 * ranges) and the backward recomputes each pixel's final transmittance and last contributor by
 * replaying the forward's front-to-back recurrence over the tile (bit-identical to the stored
 * values), saving 8 bytes per pixel for the cost of that replay.  The forward and the backward of
 * one rasterization must use the same flags.  No counterpart in the reference, which stores them
 * (ImageState, rasterizer_impl.h:48-90). */
#define OMNIGS_FLAG_RECOMPUTE_T 1

/* Inputs and outputs of one forward rasterization.
 * Replaces the argument list of CudaRasterizer::LonlatRasterizer::forward
 * (cuda_rasterizer/rasterizer.h:104-123) as called from src/rasterize_points.cu:136-155. */
typedef struct OmnigsLonlatForwardArgs {
  int P;                      /* number of Gaussians */
  int D;                      /* active SH degree, 0..3 */
  int M;                      /* SH coefficients per Gaussian (sh.size(1)); 0 without SH */
  int W, H;                   /* equirect image size */
  const float* background;    /* [3] */
  const float* means3D;       /* [P,3] */
  const float* shs;           /* [P,M,3] or NULL (then colors_precomp) */
  const float* colors_precomp;/* [P,3] or NULL */
  const float* opacities;     /* [P] */
  const float* scales;        /* [P,3] or NULL (then cov3D_precomp) */
  float scale_modifier;
  const float* rotations;     /* [P,4] or NULL */
  const float* cov3D_precomp; /* [P,6] or NULL */
  const float* viewmatrix;    /* [16] */
  const float* campos;        /* [3] */
  float* out_color;           /* [3,H,W] output */
  int* radii;                 /* [P] output */
  int flags;                  /* OMNIGS_FLAG_* (0: the reference's stored per-pixel state) */
} OmnigsLonlatForwardArgs;

/* Inputs and outputs of one backward pass.
 * Replaces CudaRasterizer::LonlatRasterizer::backward (cuda_rasterizer/rasterizer.h:126-154) as
 * called from src/rasterize_points.cu:249-276.  All outputs are fully written (zeros for
 * Gaussians with radius 0); the caller does not need to clear them. */
typedef struct OmnigsLonlatBackwardArgs {
  int P, D, M, W, H;
  int R;                      /* num_rendered of the forward, or -1 to use the device value */
  const float* background;
  const float* means3D;
  const float* shs;
  const float* colors_precomp;
  const float* scales;
  float scale_modifier;
  const float* rotations;
  const float* cov3D_precomp;
  const float* viewmatrix;
  const float* campos;
  const int* radii;           /* [P], from the forward */
  const float* dL_dout_color; /* [3,H,W] */
  float* dL_dmeans2D;         /* [P,3] (viewspace-point gradient, NDC scale, z = 0) */
  float* dL_dcolors;          /* [P,3] */
  float* dL_dopacity;         /* [P] */
  float* dL_dmeans3D;         /* [P,3] */
  float* dL_dcov3D;           /* [P,6] */
  float* dL_dsh;              /* [P,M,3] or NULL when M == 0 */
  float* dL_dscales;          /* [P,3] */
  float* dL_drotations;       /* [P,4] */
  float* dL_dconic;           /* [P,4] (x, y, 0, w) or NULL; internal in the reference */
  int flags;                  /* OMNIGS_FLAG_*, as given to the forward */
} OmnigsLonlatBackwardArgs;

/* Library version string. */
const char* omnigs_version(void);

/* Message of the last error on this host thread ("" if none). */
const char* omnigs_last_error(void);

/* Buffer sizes.  GeometryState / ImageState / BinningState sizes of the reference
 * (rasterizer_impl.h:97-102, required<T>); the binning size is a function of the capacity, the
 * largest num_rendered it can hold. */
size_t omnigs_lonlat_geom_bytes(int P);
size_t omnigs_lonlat_image_bytes(int W, int H);
/* Image buffer size for the given OMNIGS_FLAG_* bits (with OMNIGS_FLAG_RECOMPUTE_T: tile ranges only). */
size_t omnigs_lonlat_image_bytes_flags(int W, int H, int flags);
size_t omnigs_lonlat_binning_bytes(int64_t capacity);
int64_t omnigs_lonlat_binning_capacity(size_t binning_bytes);

/* Preprocess + scan (forward.cu:592-703 and rasterizer_impl.cu:622-623): writes radii and the
 * geometry buffer, including the device-side num_rendered.  No host synchronisation. */
int omnigs_lonlat_preprocess(const OmnigsLonlatForwardArgs* args, void* geom, size_t geom_bytes,
                             omnigs_stream_t stream);

/* Binning + forward blend (rasterizer_impl.cu:630-694): duplicate keys, radix sort, tile ranges,
 * blend into out_color.  Resumes from a geometry buffer filled by omnigs_lonlat_preprocess, so a
 * caller whose binning capacity was too small can resize and call this again. */
int omnigs_lonlat_render(const OmnigsLonlatForwardArgs* args, void* geom, size_t geom_bytes,
                         void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                         omnigs_stream_t stream);

/* omnigs_lonlat_preprocess followed by omnigs_lonlat_render.  Replaces
 * CudaRasterizer::LonlatRasterizer::forward (rasterizer_impl.cu:540-697) without its mid-pass
 * device-to-host copy of num_rendered (:627-628). */
int omnigs_lonlat_forward(const OmnigsLonlatForwardArgs* args, void* geom, size_t geom_bytes,
                          void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                          omnigs_stream_t stream);

/* omnigs_lonlat_forward for callers that cannot allocate device memory (a plugin inside a host
 * application that owns all device memory, or a fixed-budget real-time loop that must not call
 * cudaMalloc).  This entry point has no counterpart in the reference.  The geometry, image and
 * binning state live in a 16 MiB __device__ array inside this library (held by every GPU that
 * loads it until exit), so the caller passes only inputs and outputs.  Limits: P <= 32768,
 * W * H <= 262144 and the instances must fit the rest of the array (OMNIGS_ERR_CAPACITY
 * otherwise).  It allocates no device memory; it waits for `stream` at the end to read the status
 * and returns num_rendered.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.  Under CUDA's default
 * lazy module loading the array is reserved when this library's kernels are first used on a
 * device, which can be that first call; a caller that then reserves all remaining device memory
 * should make one early call first (P = 0 suffices) or run with CUDA_MODULE_LOADING=EAGER.  The
 * looked-up address is kept for the life of the process: do not use this entry point on a device
 * after cudaDeviceReset.  All calls share the array: calls that overlap on the GPU race and must
 * not be issued. */
int omnigs_lonlat_forward_noalloc(const OmnigsLonlatForwardArgs* args, int* num_rendered,
                                  omnigs_stream_t stream);

/* omnigs_lonlat_forward that also returns num_rendered and the status word (what
 * omnigs_lonlat_read_status gives), waiting only until the binning stage has run rather than for
 * the whole stream: the forward blend is still executing on `stream` when it returns, so the
 * caller's next launches overlap it.  Used by the LibTorch layer, whose RasterizeGaussiansCUDA
 * returns num_rendered by value (src/rasterize_points.cu:163; the reference copies it to the host
 * mid-pass, rasterizer_impl.cu:627-628).  The header is copied into pinned host memory that the
 * library creates on a thread's first call on a device (with an event) and keeps until exit; the
 * wait makes the call unsuitable for stream capture. */
int omnigs_lonlat_forward_early_status(const OmnigsLonlatForwardArgs* args, void* geom, size_t geom_bytes,
                                       void* binning, size_t binning_bytes, void* image,
                                       size_t image_bytes, int* num_rendered, uint32_t* status,
                                       omnigs_stream_t stream);

/* Waits for `stream` and copies num_rendered and the status word to the host.  The one call that
 * synchronises; the reference's forward returns num_rendered by value (rasterizer.h:104). */
int omnigs_lonlat_read_status(const void* geom, int* num_rendered, uint32_t* status,
                              omnigs_stream_t stream);

/* Backward blend + backward preprocess.  Replaces CudaRasterizer::LonlatRasterizer::backward
 * (rasterizer_impl.cu:701-795). */
int omnigs_lonlat_backward(const OmnigsLonlatBackwardArgs* args, void* geom, size_t geom_bytes,
                           const void* binning, size_t binning_bytes, const void* image,
                           size_t image_bytes, omnigs_stream_t stream);

/* ---------------------------------------------------------------- batched views -------------
 * Many equirect views of uneven resolution over one shared Gaussian set, rendered and
 * back-propagated with one launch per stage for the whole batch.  The reference renders one view
 * per call (GaussianRenderer::renderLonlat, src/gaussian_renderer.cpp:167, driven per keyframe by
 * GaussianMapper::trainForOneIteration, src/gaussian_mapper.cpp:290-440); a batch of V views
 * produces per view exactly the image of a single-view forward (same sorted instance lists, same
 * per-pixel arithmetic) and gradients equal to the sum of the V single-view backwards, summed on
 * the device instead of by V separate kernels.  The backward also accumulates the trainer's
 * densification statistics (gaussian_mapper.cpp:423-428, gaussian_model.cpp:839-853).
 *
 * State: one caller-owned buffer of omnigs_batch_state_bytes() for the per-(view, Gaussian)
 * records and per-pixel state, plus a binning buffer of omnigs_lonlat_binning_bytes(capacity) for
 * the instances of all views together.  Nothing synchronises the host except
 * omnigs_batch_read_status; a batch whose instances exceed the capacity sets
 * OMNIGS_STATUS_CAPACITY, skips binning and blending, and can be resumed with omnigs_batch_render
 * after the binning buffer is grown.  The per-view pose arrays are read on the device when the
 * kernels run, so a captured CUDA graph of these calls replays with updated poses.
 *
 * Precision options: sh_dtype OMNIGS_SH_BF16 reads SH coefficients stored as bfloat16 (colour,
 * transmittance and all gradients still accumulate in FP32; dL_dsh is FP32); fp64_poles evaluates
 * the 2D covariance, its inverse and its backward in FP64 for Gaussians beyond 85 degrees of
 * latitude in a view, where the lonlat Jacobian degenerates.  With both off, every view's image
 * and instance list are bit-identical to omnigs_lonlat_forward's. */
#define OMNIGS_MAX_BATCH_VIEWS 32
#define OMNIGS_SH_FP32 0
#define OMNIGS_SH_BF16 1

typedef struct OmnigsBatchView {
  int W, H;
  float* out_color;            /* [3,H,W] output of the forward */
  const float* dL_dout_color;  /* [3,H,W] input of the backward (unused by the forward) */
} OmnigsBatchView;

typedef struct OmnigsBatchArgs {
  int P, D, M;                 /* Gaussians, active SH degree, SH coefficients per Gaussian */
  int V;                       /* views, 1..OMNIGS_MAX_BATCH_VIEWS */
  int sh_dtype;                /* OMNIGS_SH_FP32 or OMNIGS_SH_BF16 */
  int fp64_poles;              /* 0 or 1 */
  const float* means3D;        /* [P,3] */
  const void* shs;             /* [P,M,3] fp32 or bf16, or NULL (then colors_precomp) */
  const float* colors_precomp; /* [P,3] or NULL */
  const float* opacities;      /* [P] */
  const float* scales;         /* [P,3] or NULL (then cov3D_precomp) */
  float scale_modifier;
  const float* rotations;      /* [P,4] or NULL */
  const float* cov3D_precomp;  /* [P,6] or NULL */
  const float* viewmatrices;   /* [V,16] device, each Tcw column-major as in the single-view args */
  const float* campos;         /* [V,3] device */
  const float* backgrounds;    /* [V,3] device */
  const OmnigsBatchView* views;/* [V] host array */
  int seam_wrap;               /* 0: the reference's clamped tile rects (default); 1: splats wrap
                                  across the longitude seam (cyclic tile columns, distances to the
                                  nearest copy), which removes the seam cut of the reference */
} OmnigsBatchArgs;

/* Gradient outputs of the batched backward: parameter gradients summed over the views (fully
 * written), plus optional densification statistics accumulated in place over the views where
 * the Gaussian is visible (radius > 0): grad_accum += |dL/dmean2D.xy| (viewspace-point gradient,
 * NDC scale), denom += 1, max_radii = max(max_radii, radius). */
typedef struct OmnigsBatchGrads {
  float* dL_dmeans3D;   /* [P,3] */
  float* dL_dsh;        /* [P,M,3] fp32, or NULL without SH */
  float* dL_dopacity;   /* [P] */
  float* dL_dscales;    /* [P,3] */
  float* dL_drotations; /* [P,4] */
  float* dL_dcolors;    /* [P,3] or NULL */
  float* dL_dcov3D;     /* [P,6] or NULL */
  float* grad_accum;    /* [P] or NULL */
  float* denom;         /* [P] or NULL */
  float* max_radii;     /* [P] or NULL */
} OmnigsBatchGrads;

/* Size of the batch state buffer for P Gaussians and V views of sizes W[v] x H[v] (0 if the
 * arguments are invalid). */
size_t omnigs_batch_state_bytes(int P, int V, const int* W, const int* H);

/* Preprocess of every view, then omnigs_batch_render. */
int omnigs_batch_forward(const OmnigsBatchArgs* args, void* state, size_t state_bytes, void* binning,
                         size_t binning_bytes, omnigs_stream_t stream);

/* Binning and forward blend of all views from a state filled by a preprocess (resume after a
 * capacity overflow). */
int omnigs_batch_render(const OmnigsBatchArgs* args, void* state, size_t state_bytes, void* binning,
                        size_t binning_bytes, omnigs_stream_t stream);

/* Backward blend of all views and the batched backward preprocess. */
int omnigs_batch_backward(const OmnigsBatchArgs* args, const OmnigsBatchGrads* grads, void* state,
                          size_t state_bytes, const void* binning, size_t binning_bytes,
                          omnigs_stream_t stream);

/* Splats staged per shared-memory batch in the blend kernels, per direction: 128, 256 or 512
 * (defaults: 128 forward, 128 backward).  Results do not depend on it (every pixel meets the same splats in the same order);
 * the best size depends on the scene and resolution.  Process-wide setting. */
int omnigs_set_blend_batch(int forward, int backward);
int omnigs_get_blend_batch(int* forward, int* backward);

/* Autotuner of the blend staging batch: on a batch whose forward has completed (state and
 * binning hold the sorted instance lists; every view needs out_color and dL_dout_color), times
 * the forward and backward blends of all views for each candidate size (`repeats` timed launches
 * each, CUDA events on `stream`), selects the fastest per direction with omnigs_set_blend_batch
 * and reports the times.  It synchronises the host.  The forward outputs are rewritten with
 * identical values and the gradient accumulators are cleared, so omnigs_batch_backward may follow
 * directly. */
typedef struct OmnigsTuneResult {
  int candidates[3];
  float forward_ms[3];
  float backward_ms[3];
  int forward_batch, backward_batch;
} OmnigsTuneResult;
int omnigs_batch_autotune(const OmnigsBatchArgs* args, void* state, size_t state_bytes, void* binning,
                          size_t binning_bytes, int repeats, OmnigsTuneResult* out, omnigs_stream_t stream);

/* Waits for `stream`; returns the total instance count, the per-view counts (view_rendered[V], may
 * be NULL) and the status word. */
int omnigs_batch_read_status(const void* state, int V, int64_t* num_rendered, int64_t* view_rendered,
                             uint32_t* status, omnigs_stream_t stream);

/* Failure-path check of the bounded cross-block waits (no counterpart in the reference): runs
 * omnigs_lonlat_preprocess and the binning up to the duplicate pass with scan tile 0 taken by no
 * block, so tile 1's look-back waits on a prefix that is never published; the wait gives up after
 * max_spins polls, sets OMNIGS_STATUS_LOOKBACK and the kernel finishes.  Then waits for `stream`,
 * returns the status word in *status and OMNIGS_ERR_DEVICE when a bit other than capacity is set.
 * The buffers hold no valid forward afterwards; a following omnigs_lonlat_forward resets them.
 * Needs P > 1024.  For tests: real passes never skip a tile. */
int omnigs_debug_lookback_timeout(const OmnigsLonlatForwardArgs* args, void* geom, size_t geom_bytes,
                                  void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                                  int max_spins, uint32_t* status, omnigs_stream_t stream);

/* Device pointers into the batch state, for inspection and parity testing.  Pixels of view v start
 * at pixel_base[v] of final_T / n_contrib, its tiles at tile_base[v] of ranges. */
typedef struct OmnigsBatchStateView {
  const int* radii;             /* [V][P] */
  const float* splat;           /* [V][P][8] */
  const float* color;           /* [V][P][4] */
  const float* final_T;         /* [pixels] */
  const uint32_t* n_contrib;    /* [pixels] */
  const uint32_t* ranges;       /* [tiles][2] */
  int64_t pixel_base[OMNIGS_MAX_BATCH_VIEWS];
  int64_t tile_base[OMNIGS_MAX_BATCH_VIEWS];
  int tile_passes;              /* tile-sort passes: the sorted list is in buffer (tile_passes & 1) */
  const float* depth;           /* [V][P] radial distance (the sort key's depth bits) */
} OmnigsBatchStateView;
int omnigs_batch_state_view(const void* state, int P, int V, const int* W, const int* H,
                            OmnigsBatchStateView* out);

/* ---------------------------------------------------------------- training step --------------
 * The kernels around the rasterizer in the reference's training iteration
 * (GaussianMapper::trainForOneIteration, src/gaussian_mapper.cpp:384-432).
 *
 * L1 + D-SSIM loss with its image gradient (include/loss_utils.h:30-131): for images [C,H,W],
 * using rows [0, rows) (the reference's skip-bottom slice, gaussian_mapper.cpp:389-398; rows = H
 * for the whole image), writes loss[0] = (1 - lambda) L1 + lambda (1 - SSIM), loss[1] = L1,
 * loss[2] = SSIM (device floats) and dL_dimage (zero in rows >= `rows`).  SSIM uses the
 * reference's 11x11 Gaussian window (sigma 1.5), zero padding and C1 = 0.01^2, C2 = 0.03^2.  The
 * workspace is caller-owned device memory of omnigs_l1_dssim_workspace_bytes(C, H, W). */
size_t omnigs_l1_dssim_workspace_bytes(int C, int H, int W);
int omnigs_l1_dssim(const float* image, const float* gt, int C, int H, int W, int rows, float lambda_dssim,
                    float* dL_dimage, float* loss, void* workspace, size_t workspace_bytes,
                    omnigs_stream_t stream);

/* Raw (optimised) Gaussian parameters (GaussianModel, src/gaussian_model.cpp:54-77). */
typedef struct OmnigsGaussianParams {
  int P, M;              /* Gaussians; SH coefficients per Gaussian (1 DC + M - 1 rest), M <= 16 */
  float* xyz;            /* [P,3] */
  float* features_dc;    /* [P,1,3] */
  float* features_rest;  /* [P,M-1,3] */
  float* opacity;        /* [P,1], before the sigmoid */
  float* scaling;        /* [P,3], log of the scales */
  float* rotation;       /* [P,4], quaternion (r, x, y, z) before normalisation */
} OmnigsGaussianParams;

/* Adam first and second moments, one pair per parameter array (same shapes). */
typedef struct OmnigsAdamState {
  float *m_xyz, *v_xyz, *m_dc, *v_dc, *m_rest, *v_rest, *m_opacity, *v_opacity;
  float *m_scaling, *v_scaling, *m_rotation, *v_rotation;
} OmnigsAdamState;

/* Activated values the rasterizer reads: means3D (may alias xyz), SH [P,M,3] as fp32 or bf16
 * (shs_bf16 = 1), sigmoid(opacity), exp(scaling), normalize(rotation). */
typedef struct OmnigsActivated {
  float* means3D;
  void* shs;
  int shs_bf16;
  float* opacities;
  float* scales;
  float* rotations;
} OmnigsActivated;

/* Adam hyper-parameters in DEVICE memory, read when the kernel runs (so a captured graph replays
 * with the caller's updated step and learning rates).  lr[] per parameter group in the
 * reference's order (gaussian_model.cpp:534-541): xyz, f_dc, f_rest, opacity, scaling, rotation.
 * The values are doubles, as torch's AdamOptions holds them: the kernel forms the float
 * coefficients beta, 1 - beta, lr / (1 - beta1^step) and sqrt(1 - beta2^step) in double and rounds
 * them once, as torch does.  step is the 1-based step count of the bias corrections. */
typedef struct OmnigsAdamHyper {
  double lr[6];
  double beta1, beta2, eps;
  int64_t step;
} OmnigsAdamHyper;

/* Writes the activated values of `params` (the first forward of a run). */
int omnigs_activate(const OmnigsGaussianParams* params, const OmnigsActivated* act, omnigs_stream_t stream);

/* One Adam step of every parameter group (torch::optim::Adam as set up at
 * gaussian_model.cpp:485-518, no weight decay) from the rasterizer's gradients with respect to
 * the activated values, with the activation backward fused in; then refreshes `act`.  `act` must
 * hold the activation of the current parameters (omnigs_activate or the previous step). */
int omnigs_adam_step(const OmnigsGaussianParams* params, const OmnigsAdamState* state, const OmnigsActivated* act,
                     const float* dL_dmeans3D, const float* dL_dsh, const float* dL_dopacity,
                     const float* dL_dscales, const float* dL_drotations, const OmnigsAdamHyper* hyper,
                     omnigs_stream_t stream);

/* Visibility marks.  camera_type 3: every Gaussian (markAllVisible, rasterizer_impl.cu:82-90);
 * camera_type 1: the pinhole near test p_view.z > 0.2 (checkFrustum, rasterizer_impl.cu:66-78,
 * auxiliary.h:166-196).  present is a [P] byte array. */
int omnigs_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                        uint8_t* present, omnigs_stream_t stream);

/* Per-stage device timing.  While enabled, every kernel this library launches is bracketed by
 * CUDA events recorded on its launch stream; omnigs_timing_read waits for the recorded events and
 * returns the summed device time and launch count per stage since the last read.  Disabled by
 * default (no events are recorded).  The reference has only host chrono timing
 * (src/gaussian_mapper.cpp:293, 738-781). */
#define OMNIGS_STAGE_PREPROCESS 0
#define OMNIGS_STAGE_DUPLICATE 1
#define OMNIGS_STAGE_SORT 2
#define OMNIGS_STAGE_RANGES 3
#define OMNIGS_STAGE_RENDER_FORWARD 4
#define OMNIGS_STAGE_RENDER_BACKWARD 5
#define OMNIGS_STAGE_PREPROCESS_BACKWARD 6
#define OMNIGS_STAGE_OTHER 7
#define OMNIGS_NUM_STAGES 8
typedef struct OmnigsStageTimes {
  double ms[OMNIGS_NUM_STAGES];
  uint64_t launches[OMNIGS_NUM_STAGES];
} OmnigsStageTimes;
int omnigs_timing_enable(int enable);
int omnigs_timing_read(OmnigsStageTimes* out);

/* Number of kernels this library has launched since it was loaded. */
uint64_t omnigs_kernel_launches(void);

/* Read-only views into the private buffers, for inspection and parity testing.  Pointers are
 * device pointers inside the given buffers. */
typedef struct OmnigsLonlatGeomView {
  const float* splat;          /* [P][8]: x, y, conic a, conic b, conic c, opacity, cull threshold, conic det */
  const float* color;          /* [P][4]: r, g, b, clamp bits (as uint32) */
  const float* depth;          /* [P] radial distance r (+inf where culled) */
  const uint32_t* tiles_touched; /* [P] */
  const uint32_t* depth_order; /* [P] Gaussian indices sorted by (depth bits, index) */
} OmnigsLonlatGeomView;
/* The sorted instance list: instance i covers tile tile_ids[i] and Gaussian point_list[i]; the
 * reference's 64-bit key of instance i is tile_ids[i] << 32 | float_bits(depth[point_list[i]]). */
typedef struct OmnigsLonlatBinningView {
  const uint32_t* tile_ids;    /* [num_rendered] sorted tile ids */
  const uint32_t* point_list;  /* [num_rendered] sorted Gaussian indices */
} OmnigsLonlatBinningView;
typedef struct OmnigsLonlatImageView {
  const float* final_T;     /* [H*W] */
  const uint32_t* n_contrib;/* [H*W] last contributor (1-based position in the tile range) */
  const uint32_t* ranges;   /* [tiles][2] */
} OmnigsLonlatImageView;
int omnigs_lonlat_geom_view(const void* geom, int P, OmnigsLonlatGeomView* out);
int omnigs_lonlat_binning_view(const void* binning, size_t binning_bytes, int W, int H,
                               OmnigsLonlatBinningView* out);
int omnigs_lonlat_image_view(const void* image, int W, int H, OmnigsLonlatImageView* out);
/* The batch's sorted instance list in its binning buffer, after a forward: instance i covers global
 * tile tile_ids[i] (view v owns tiles [tile_base[v], tile_base[v] + its tiles)) and splat record
 * point_list[i] = v * P + Gaussian index.  No counterpart in the reference (inspection). */
int omnigs_batch_binning_view(const void* binning, size_t binning_bytes, int P, int V, const int* W,
                              const int* H, OmnigsLonlatBinningView* out);

#ifdef __cplusplus
}
#endif

#endif /* OMNIGS_B200_H_ */
