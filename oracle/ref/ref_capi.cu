// TEST INFRASTRUCTURE ONLY.  extern "C" driver of the reference rasterizer
// (CudaRasterizer::LonlatRasterizer, cuda_rasterizer/rasterizer.h:96-155), compiled together with
// the reference's own cuda_rasterizer/*.cu from their place in the reference checkout (see
// oracle/ref/Makefile).  It stands in for src/rasterize_points.cu:133-157 / 244-277 (which needs
// LibTorch): the three state buffers grow with cudaMalloc like the reference's resized tensors, and
// ref_state() exposes the reference's own intermediate arrays for bit-exact comparison.
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>

#include "cuda_rasterizer/config.h"
#include "cuda_rasterizer/rasterizer.h"
#include "cuda_rasterizer/rasterizer_impl.h"

namespace {

struct Growable {
  char* ptr = nullptr;
  size_t cap = 0;
  char* get(size_t n) {
    if (n > cap) {
      if (ptr) cudaFree(ptr);
      ptr = nullptr;
      cudaMalloc(&ptr, n);
      cap = n;
    }
    return ptr;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct RefState {
  Growable geom, binning, img, dpx, dpy;
  int P = 0, W = 0, H = 0, R = 0;
};

}  // namespace

struct RefStateView {
  const uint32_t* tiles_touched;
  const uint32_t* point_offsets;
  const float* depths;
  const float* means2D;        // [P][2]
  const float* conic_opacity;  // [P][4]
  const float* rgb;            // [P][3]
  const uint8_t* clamped;      // [P][3]
  const float* cov3D;          // [P][6]
  const uint64_t* keys;        // [R] sorted
  const uint32_t* point_list;  // [R] sorted
  const uint64_t* keys_unsorted;
  const uint32_t* point_list_unsorted;
  const uint32_t* ranges;      // [tiles][2]
  const uint32_t* n_contrib;   // [H*W]
  const float* accum_alpha;    // [H*W] (final transmittance)
};

extern "C" {

void* ref_create() { return new RefState(); }

void ref_destroy(void* h) {
  auto* s = static_cast<RefState*>(h);
  s->geom.release();
  s->binning.release();
  s->img.release();
  s->dpx.release();
  s->dpy.release();
  delete s;
}

int ref_forward(void* h, int P, int D, int M, const float* background, int W, int H, const float* means3D,
                const float* shs, const float* colors_precomp, const float* opacities, const float* scales,
                float scale_modifier, const float* rotations, const float* cov3D_precomp,
                const float* viewmatrix, const float* campos, float* out_color, int* radii) {
  auto* s = static_cast<RefState*>(h);
  std::function<char*(size_t)> gf = [s](size_t n) { return s->geom.get(n); };
  std::function<char*(size_t)> bf = [s](size_t n) { return s->binning.get(n); };
  std::function<char*(size_t)> imf = [s](size_t n) { return s->img.get(n); };
  const int R = CudaRasterizer::LonlatRasterizer::forward(gf, bf, imf, P, D, M, background, W, H, means3D, shs,
                                                          colors_precomp, opacities, scales, scale_modifier,
                                                          rotations, cov3D_precomp, viewmatrix, campos, false,
                                                          out_color, radii);
  s->P = P;
  s->W = W;
  s->H = H;
  s->R = R;
  return R;
}

// Gradient outputs must be zero-filled by the caller (the reference allocates them with
// torch::zeros, src/rasterize_points.cu:200-208).
void ref_backward(void* h, int D, int M, const float* background, const float* means3D, const float* shs,
                  const float* colors_precomp, const float* scales, float scale_modifier, const float* rotations,
                  const float* cov3D_precomp, const float* viewmatrix, const float* campos, const int* radii,
                  const float* dL_dpix, float* dL_dmean2D, float* dL_dconic, float* dL_dopacity,
                  float* dL_dcolor, float* dL_dmean3D, float* dL_dcov3D, float* dL_dsh, float* dL_dscale,
                  float* dL_drot) {
  auto* s = static_cast<RefState*>(h);
  float* dpx = reinterpret_cast<float*>(s->dpx.get(sizeof(float) * 3 * (size_t)s->P));
  float* dpy = reinterpret_cast<float*>(s->dpy.get(sizeof(float) * 3 * (size_t)s->P));
  cudaMemset(dpx, 0, sizeof(float) * 3 * (size_t)s->P);
  cudaMemset(dpy, 0, sizeof(float) * 3 * (size_t)s->P);
  CudaRasterizer::LonlatRasterizer::backward(s->P, D, M, s->R, background, s->W, s->H, means3D, shs,
                                             colors_precomp, scales, scale_modifier, rotations, cov3D_precomp,
                                             viewmatrix, campos, radii, s->geom.ptr, s->binning.ptr, s->img.ptr,
                                             dL_dpix, dL_dmean2D, dL_dconic, dL_dopacity, dL_dcolor, dL_dmean3D,
                                             dL_dcov3D, dL_dsh, dL_dscale, dL_drot, dpx, dpy);
}

// Device-to-device copy used to export the reference's arrays.
int ref_copy(void* dst, const void* src, size_t nbytes) {
  return (int)cudaMemcpy(dst, src, nbytes, cudaMemcpyDeviceToDevice);
}

int ref_state(void* h, RefStateView* out) {
  auto* s = static_cast<RefState*>(h);
  char* g = s->geom.ptr;
  char* b = s->binning.ptr;
  char* im = s->img.ptr;
  auto geom = CudaRasterizer::GeometryState::fromChunk(g, s->P);
  auto bin = CudaRasterizer::BinningState::fromChunk(b, s->R);
  auto img = CudaRasterizer::ImageState::fromChunk(im, (size_t)s->W * s->H);
  out->tiles_touched = geom.tiles_touched;
  out->point_offsets = geom.point_offsets;
  out->depths = geom.depths;
  out->means2D = reinterpret_cast<const float*>(geom.means2D);
  out->conic_opacity = reinterpret_cast<const float*>(geom.conic_opacity);
  out->rgb = geom.rgb;
  out->clamped = reinterpret_cast<const uint8_t*>(geom.clamped);
  out->cov3D = geom.cov3D;
  out->keys = bin.point_list_keys;
  out->point_list = bin.point_list;
  out->keys_unsorted = bin.point_list_keys_unsorted;
  out->point_list_unsorted = bin.point_list_unsorted;
  out->ranges = reinterpret_cast<const uint32_t*>(img.ranges);
  out->n_contrib = img.n_contrib;
  out->accum_alpha = img.accum_alpha;
  return s->R;
}

}  // extern "C"
