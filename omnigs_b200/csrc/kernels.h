// Internal launch interface between the C-ABI (capi.cu) and the kernels.  No torch types.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "layout.h"

namespace omnigs {


struct PreprocessParams {
  int P, D, M, W, H, gx, gy;
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* opacities;
  const float* shs;
  const float* colors_precomp;
  const float* cov3D_precomp;
  float scale_modifier;
  const float* viewmatrix;
  const float* campos;
  int* radii;
  float4* splat;
  float4* color;
  float* depth;              // [P] radial depth; +inf for culled Gaussians (depth-sort key)
  uint32_t* tiles_touched;   // [P]
  float4* grad_acc;
  GeomHeader* hdr;           // num_rendered64 is accumulated here
};

// Digit histograms of up to kDepthPasses digits of u32 keys.
// With seg_len > 0 the keys are num_segs independent segments of seg_len items each (the views of
// a batch) and every segment gets its own histograms, at hist + seg * passes * kRadix.
struct HistParams {
  const uint32_t* keys;
  uint32_t n_host;             // item count when count_hdr is null
  const GeomHeader* count_hdr; // else the device num_rendered (0 if over capacity)
  int64_t capacity;
  int passes;
  int shift[kDepthPasses];
  uint32_t mask[kDepthPasses];
  uint32_t* hist;              // [segments][passes][kRadix], zeroed by the caller
  uint32_t seg_len;            // 0: one segment of all items
  uint32_t num_segs;
};

// One stable LSD radix pass over (u32 key, u32 value) pairs.
struct OnesweepParams {
  const uint32_t* keys_in;
  const uint32_t* vals_in;     // null: the value is the item index
  uint32_t* keys_out;
  uint32_t* vals_out;
  int shift;
  uint32_t mask;
  uint32_t n_host;
  const GeomHeader* count_hdr;
  int64_t capacity;
  const uint32_t* hist;        // this pass's [kRadix] histogram (of segment 0)
  uint32_t* lookback;          // [sort tiles][kRadix], zeroed by the caller
  uint32_t* tile_counter;      // zeroed by the caller
  GeomHeader* hdr;             // status bits
  // Segmented sort (each segment sorted on its own, in place): seg_len items per segment, the
  // histogram of segment s at hist + s * hist_seg_stride.  seg_len == 0: one segment.
  uint32_t seg_len;
  uint32_t num_segs;
  uint32_t hist_seg_stride;
  // Variable segments (seg_counts non-null): num_segs consecutive segments of seg_counts[s] items
  // (device counts, all taken as 0 when count_hdr reports an overflow) with segment-local keys;
  // with add_key_base the pass writes key + (segment s's key base) (the last pass restores global
  // keys).  The key bases are the u32[kMaxBatchViews] array that directly follows the
  // u64[kMaxBatchViews] counts (BatchLayout), so this parameter block stays at 128 bytes: at 136
  // bytes every launch of the pass measured ~2 us slower on a B200.
  const unsigned long long* seg_counts;
  int add_key_base;
};

// duplicateWithKeys over V views (V = 1 for a single view).  Records are view-major (rec = v P + g);
// instance keys are global tile ids tile_base[v] + ty gx[v] + tx and values record indices.
struct DuplicateParams {
  int P, V;
  const int* radii;            // [V][P]
  const float4* splat;         // [V][P][2]
  const uint32_t* order;       // [V][P] record indices sorted by (view, depth bits, index)
  uint32_t* tkeys;             // [capacity] tile ids
  uint32_t* tvals;             // [capacity] record indices
  unsigned long long* scan_state;
  uint32_t* incl;              // [V][P] scratch: inclusive instance offsets in depth order
                               // (the depth sort's first key buffer, free after its last pass)
  // [V][P] scratch in depth order, written by the scan for the emission: each Gaussian's first
  // row's tile id and its first column | width << 16 (the depth sort's free buffers)
  uint32_t* rect_row;
  uint32_t* rect_cw;
  uint32_t* emit_first;        // [emit_blocks(capacity) + 1]: depth-order position of the Gaussian
  uint32_t* emit_last;         // holding each emit block's first / last instance
  int64_t capacity;
  GeomHeader* hdr;
  int seam_wrap;               // tile columns wrap modulo gx (rects from tile_rect_cyclic)
  int gx[kMaxBatchViews], gy[kMaxBatchViews];
  uint32_t tile_base[kMaxBatchViews];
  // digit histograms of the tile sort, accumulated into hist[hist_passes][kRadix] (zeroed by the
  // caller); hist_passes 0 counts nothing.  With hist_per_view, the keys written are view-local
  // tile ids (without tile_base[v]) and each view's digits are counted into
  // hist + v * kTilePasses * kRadix (requires P >= kScanBlock: a block then spans at most two views).
  uint32_t* hist;
  int hist_passes;
  int hist_shift[kTilePasses];
  uint32_t hist_mask[kTilePasses];
  int hist_per_view;
  uint32_t* key_base_out;      // with hist_per_view: tile_base[0, V) copied here for the tile sort
  // Look-back wait limit (polls; 0 = kMaxSpins) and the number of leading scan tiles no block
  // takes (0 in every real pass).  omnigs_debug_lookback_timeout sets skip_tiles = 1 and a small
  // limit: tile 0 then never publishes its prefix, so tile 1's bounded wait runs out.
  int max_spins;
  uint32_t skip_tiles;
};

struct RangesParams {
  const uint32_t* keys;        // sorted tile ids
  uint2* ranges;
  uint32_t num_tiles;
  int64_t capacity;
  const GeomHeader* hdr;
};

struct RenderParams {
  int P, W, H, gx, gy;
  const uint2* ranges;
  const uint32_t* point_list;
  int64_t capacity;
  const float4* splat;
  const float4* color;
  const float* bg;
  float* out_color;
  float* final_T;       // NULL with transmittance checkpointing: the forward does not store it and
  uint32_t* n_contrib;  // the backward recomputes it
  // backward only
  const float* dL_dpix;
  float* grad_acc;  // [P][12]
};

struct PreprocessBackwardParams {
  int P, D, M, W, H;
  const float* means3D;
  const int* radii;
  const float* shs;
  const float4* color;  // clamp bits in .w
  const float4* splat;  // [P][2] splat records (their conic turns the blend's mean sums into terms)
  const float* scales;
  const float* rotations;
  const float* cov3D_precomp;
  float scale_modifier;
  const float* viewmatrix;
  const float* campos;
  float4* grad_acc;     // consumed and cleared
  float* dL_dmeans2D;   // [P,3]
  float* dL_dconic;     // [P,4] or null
  float* dL_dopacity;   // [P]
  float* dL_dcolors;    // [P,3]
  float* dL_dmeans3D;   // [P,3]
  float* dL_dcov3D;     // [P,6]
  float* dL_dsh;        // [P,M,3] or null
  float* dL_dscales;    // [P,3]
  float* dL_drotations; // [P,4]
};

// ------------------------------------------------------------------ batched views -------------
// Many equirect views of one shared Gaussian set.  Per-(view, Gaussian) records are view-major:
// record index rec = v * P + g.  Global tile ids run over all views: view v owns
// [tile_base, tile_base + gx * gy); its pixels occupy [pixel_base, pixel_base + W * H) of the
// per-pixel state arrays.
struct BatchView {
  int W, H, gx, gy;
  uint32_t tile_base;
  uint32_t pixel_base;
  float* out_color;             // [3,H,W]
  const float* dL_dpix;         // [3,H,W] (backward)
};

struct BatchParams {
  int P, V, D, M;
  int sh_bf16;                  // shs holds bf16 instead of fp32 values
  int seam_wrap;                // cyclic tile columns and wrapped blend distance
  uint32_t total_tiles;
  const float* means3D;
  const float* scales;
  const float* rotations;
  const float* opacities;
  const void* shs;
  const float* colors_precomp;
  const float* cov3D_precomp;
  float scale_modifier;
  const float* viewmatrices;    // [V][16]
  const float* campos;          // [V][3]
  const float* backgrounds;     // [V][3]
  int* radii;                   // [V][P]
  float4* splat;                // [V][P][2]
  float4* color;                // [V][P]
  float* depth;                 // [V][P]
  float4* grad_acc;             // [V][P][3]
  GeomHeader* hdr;
  unsigned long long* view_rendered;  // [V] instances per view
  BatchView views[kMaxBatchViews];
};

// Gradient outputs of the batched backward, summed over the views, plus the densification
// statistics the trainer accumulates per view (gaussian_mapper.cpp:423-428,
// gaussian_model.cpp:839-853).  Every non-null output is fully written, except the statistics,
// which are accumulated into.
struct BatchGrads {
  float* dL_dmeans3D;    // [P,3]
  float* dL_dsh;         // [P,M,3] fp32 (null when there are no SH)
  float* dL_dopacity;    // [P]
  float* dL_dscales;     // [P,3]
  float* dL_drotations;  // [P,4]
  float* dL_dcolors;     // [P,3] or null (precomputed colours)
  float* dL_dcov3D;      // [P,6] or null (precomputed covariances)
  float* grad_accum;     // [P] += |dL/dmean2D.xy| per view where visible, or null
  float* denom;          // [P] += 1 per view where visible, or null
  float* max_radii;      // [P] = max(max_radii, radius) over visible views, or null
};


struct BatchRenderParams {
  int P, V;
  const uint2* ranges;          // [total tiles]
  const uint32_t* point_list;   // record indices
  int64_t capacity;
  const float4* splat;
  const float4* color;
  const float* backgrounds;     // [V][3]
  float* final_T;               // [total pixels]
  uint32_t* n_contrib;          // [total pixels]
  float* grad_acc;              // [V][P][12]
  uint32_t total_tiles;
  int seam_wrap;                // blend distances to the splat copy nearest each warp patch
  BatchView views[kMaxBatchViews];
  uint8_t tile_order[kMaxBatchViews];  // view indices by ascending tile_base
};

void launch_batch_preprocess(const BatchParams& p, int fp64_poles, cudaStream_t s);
void launch_batch_render_forward(const BatchRenderParams& p, cudaStream_t s);
void launch_batch_render_backward(const BatchRenderParams& p, cudaStream_t s);
void launch_batch_preprocess_backward(const BatchParams& p, const BatchGrads& g, int fp64_poles,
                                      cudaStream_t s);

void launch_preprocess(const PreprocessParams& p, cudaStream_t s);
void launch_histogram(const HistParams& p, int64_t max_items, cudaStream_t s);
void launch_onesweep(const OnesweepParams& p, int64_t max_items, cudaStream_t s);
void launch_duplicate(const DuplicateParams& p, cudaStream_t s);
void launch_ranges(const RangesParams& p, cudaStream_t s);
// Splats staged per shared-memory batch in the blend kernels: a template parameter chosen at run
// time per direction (128, 256 or 512; set by omnigs_set_blend_batch or the autotuner).  Results
// do not depend on it: every pixel meets the same splats in the same order.  Defaults: 128 for both
// directions (the faster of the three for each on the 1M-Gaussian 2048x1024 view on a B200:
// forward 0.512 vs 0.522 ms at 256, backward 1.149 vs 1.163 ms at 256).
constexpr int kDefaultBatch = 128;
constexpr int kDefaultBwdBatch = 128;
int blend_batch_size(bool backward);

void launch_render_forward(const RenderParams& p, cudaStream_t s);
void launch_render_backward(const RenderParams& p, cudaStream_t s);
void launch_preprocess_backward(const PreprocessBackwardParams& p, cudaStream_t s);

// Sets the message returned by omnigs_last_error() on this host thread.
void set_last_error(const char* msg);

void launch_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                         bool* present, cudaStream_t s);

}  // namespace omnigs
