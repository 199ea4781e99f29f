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
struct HistParams {
  const uint32_t* keys;
  uint32_t n_host;             // item count when count_hdr is null
  const GeomHeader* count_hdr; // else the device num_rendered (0 if over capacity)
  int64_t capacity;
  int passes;
  int shift[kDepthPasses];
  uint32_t mask[kDepthPasses];
  uint32_t* hist;              // [passes][kRadix], zeroed by the caller
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
  const uint32_t* hist;        // this pass's [kRadix] histogram
  uint32_t* lookback;          // [sort tiles][kRadix], zeroed by the caller
  uint32_t* tile_counter;      // zeroed by the caller
  GeomHeader* hdr;             // status bits
};

struct DuplicateParams {
  int P, gx, gy;
  const int* radii;
  const float4* splat;
  const uint32_t* order;       // [P] Gaussian indices sorted by (depth bits, index)
  uint32_t* tkeys;             // [capacity] tile ids
  uint32_t* tvals;             // [capacity] Gaussian indices
  unsigned long long* scan_state;
  int64_t capacity;
  GeomHeader* hdr;
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
  float* final_T;
  uint32_t* n_contrib;
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

void launch_preprocess(const PreprocessParams& p, cudaStream_t s);
void launch_histogram(const HistParams& p, int64_t max_items, cudaStream_t s);
void launch_onesweep(const OnesweepParams& p, int64_t max_items, cudaStream_t s);
void launch_duplicate(const DuplicateParams& p, cudaStream_t s);
void launch_ranges(const RangesParams& p, cudaStream_t s);
void launch_render_forward(const RenderParams& p, cudaStream_t s);
void launch_render_backward(const RenderParams& p, cudaStream_t s);
void launch_preprocess_backward(const PreprocessBackwardParams& p, cudaStream_t s);

// Sets the message returned by omnigs_last_error() on this host thread.
void set_last_error(const char* msg);

void launch_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                         bool* present, cudaStream_t s);

}  // namespace omnigs
