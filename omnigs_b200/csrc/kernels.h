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
  float* depth;
  uint32_t* offsets;
  float4* grad_acc;
  unsigned long long* scan_state;
  GeomHeader* hdr;
};

struct DuplicateParams {
  int P, gx, gy, passes, last_pass_bits;
  const int* radii;
  const float4* splat;
  const float* depth;
  const uint32_t* offsets;
  uint64_t* keys;
  uint32_t* vals;
  uint32_t* hist;      // [kMaxSortPasses][kRadix], zeroed by the caller
  uint32_t* lookback;  // [kMaxSortPasses][sort tiles][kRadix], cleared here for the tiles in use
  int64_t lookback_pass_stride;
  int64_t capacity;
  GeomHeader* hdr;
};

struct SortPassParams {
  const uint64_t* keys_in;
  const uint32_t* vals_in;
  uint64_t* keys_out;
  uint32_t* vals_out;
  const uint32_t* hist;   // this pass's [kRadix] digit histogram
  uint32_t* lookback;     // this pass's [sort tiles][kRadix] look-back words
  uint32_t* tile_counter;
  int shift;
  int64_t capacity;
  GeomHeader* hdr;        // reads num_rendered / status, sets status bits
};

struct RangesParams {
  const uint64_t* keys;
  uint2* ranges;
  uint32_t num_tiles;
  int64_t capacity;
  GeomHeader* hdr;
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
void launch_duplicate(const DuplicateParams& p, cudaStream_t s);
void launch_sort_pass(const SortPassParams& p, cudaStream_t s);
void launch_ranges(const RangesParams& p, cudaStream_t s);
void launch_render_forward(const RenderParams& p, cudaStream_t s);
void launch_render_backward(const RenderParams& p, cudaStream_t s);
void launch_preprocess_backward(const PreprocessBackwardParams& p, cudaStream_t s);
// Sets the message returned by omnigs_last_error() on this host thread.
void set_last_error(const char* msg);

void launch_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                         bool* present, cudaStream_t s);

}  // namespace omnigs
