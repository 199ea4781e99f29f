// Per-(view, Gaussian) body of the forward lonlat preprocess, shared by the single-view kernel and
// the batched multi-view kernel.
//
// Evaluates the reference's FP32 sequence (forward.cu:592-703): near cull at r^2 <= 0.04,
// equirect projection, 2D covariance through the lonlat Jacobian, conic, radius, clamped tile rect
// and SH colour.  Besides the reference's outputs, each visible splat gets the threshold of its
// quadratic form beyond which its alpha is provably below 1/255, and the conic's determinant; the
// blend kernels use them to skip a splat for a whole warp without changing any per-pixel decision.
#pragma once

#include "device_util.cuh"
#include "lonlat_math.cuh"

namespace omnigs {

// Alpha-support quadric of a splat: {thr, det} such that o * exp(power) can reach the reference's
// 1/255 skip threshold (forward.cu:436-438) only where d^T Q d <= thr, Q = [a b; b c] the conic and
// d = centre - pixel (power = -d^T Q d / 2).  Exactly, alpha >= 1/255 needs d^T Q d <= 2 tau with
// tau = ln(255 o); thr adds 0.01 to tau (expf error, FP32 rounding of `power`) and a relative
// 1e-5 a c / det, which grows with the ellipse's elongation like the cancellation error of the
// blends' FP32 evaluation of `power` (its terms reach 2 tau a c / det on the ellipse), rounded up.
// det = a c - b^2 is exact in FP64 from the float conic and rounded down.  Both err towards "the
// splat may contribute".  Non-finite inputs or a conic that is not positive definite give
// det = NaN (every patch test hits: the per-pixel test decides); an opacity that can never reach
// 1/255 gives thr = -inf (no patch test hits).
__device__ __forceinline__ float2 cull_quadric(float x, float y, float a, float b, float c, float o) {
  const float inf = __int_as_float(0x7f800000), nan = __int_as_float(0x7fffffff);
  if (!(isfinite(x) && isfinite(y) && isfinite(a) && isfinite(b) && isfinite(c) && isfinite(o)))
    return make_float2(inf, nan);
  if (!(o > 0.0f)) return make_float2(-inf, 1.0f);
  const double tau = log(255.0 * (double)o) + 0.01;
  if (tau <= 0.0) return make_float2(-inf, 1.0f);
  const double A = a, B = b, C = c;
  const double det = A * C - B * B;
  if (!(A > 0.0) || !(C > 0.0) || !(det > 0.0)) return make_float2(inf, nan);
  const double thr = 2.0 * tau * (1.0 + 1e-5 * (A * C / det));
  return make_float2(__double2float_ru(thr), __double2float_rd(det));
}

// One splat of one view.  radius == 0 means culled; then only depth_key (+inf, so culled
// Gaussians sort last) and touched (0) are meaningful.
struct SplatResult {
  int radius;
  uint32_t touched;
  float depth_key;
  float4 s0;   // x, y, conic a, conic b
  float4 s1;   // conic c, opacity, cull threshold, conic determinant
  float4 col;  // r, g, b, clamp bits
};

// |latitude| above which the precision mode evaluates the 2D covariance in FP64: 85 degrees,
// where the lonlat Jacobian's longitude row (~ W / (2 pi rho)) has grown ~11x over the equator's.
constexpr float kPoleSinLat = 0.99619469809174553f;  // sin(85 deg)

// cov3d(out) fills the Gaussian's 3D covariance; it is called after the near cull and before a
// compiler barrier, as the reference stores cov3D to global memory at that point (forward.cu:650)
// and its 2D-covariance code then reloads the view matrix and recomputes the camera-space mean
// instead of reusing the values above.  The barrier keeps that dataflow (and therefore the same
// FMA contraction), so radii and tile rects stay bit-identical.  `vm` must point to memory (not
// registers) for the reload to happen.  sh(k) returns coefficient k as a V3.
// seam_wrap selects the cyclic tile-column range (tile_rect_cyclic) instead of the clamped one.
// With kFp64Poles, Gaussians beyond kPoleSinLat get their 2D covariance, conic and radius from an
// FP64 evaluation of the same formulas (not the reference's arithmetic: a precision mode).
template <bool kFp64Poles, class Cov3DFn, class ShLoad>
__device__ __forceinline__ SplatResult preprocess_splat(float3 p_orig, const float* vm, int W, int H,
                                                        int gx, int gy, int D, const float* campos,
                                                        float opacity, const float* color_precomp,
                                                        bool seam_wrap, Cov3DFn cov3d, ShLoad sh) {
  SplatResult res;
  res.radius = 0;
  res.touched = 0;
  res.depth_key = __int_as_float(0x7f800000);
  // near cull, auxiliary.h:198-220 (no frustum test for lonlat)
  const float3 p_view = xform_point(p_orig, vm);
  const float rr = p_view.x * p_view.x + p_view.y * p_view.y + p_view.z * p_view.z;
  if (rr <= 0.04f) return res;
  const float r = sqrtf(rr);
  // point3ToLonlatScreen, auxiliary.h:236-248
  const float inv_r = 1.0f / (r + 0.0000001f);
  const float lon = atan2f(p_view.x, p_view.z);
  const float lat = asinf(p_view.y * inv_r);
  const float scr_x = lon * kInvPi;
  const float scr_y = lat * kTwoInvPi;
  float cov3D[6];
  cov3d(cov3D);
  asm volatile("" ::: "memory");
  float3 conic;
  float my_radius;
  if (kFp64Poles && fabsf(p_view.y) > kPoleSinLat * r) {
    double3 cov = cov2d_lonlat_f64(p_orig, W, H, cov3D, vm);
    const double det = cov.x * cov.z - cov.y * cov.y;
    if (!(det > 0.0)) return res;
    const double det_inv = 1.0 / det;
    conic = make_float3((float)(cov.z * det_inv), (float)(-cov.y * det_inv), (float)(cov.x * det_inv));
    const double mid = 0.5 * (cov.x + cov.z);
    const double lambda1 = mid + sqrt(fmax(0.1, mid * mid - det));
    my_radius = (float)ceil(3.0 * sqrt(lambda1));
  } else {
    const float3 cov = cov2d_lonlat(p_orig, W, H, cov3D, vm);
    const float det = (cov.x * cov.z - cov.y * cov.y);
    if (det == 0.0f) return res;
    const float det_inv = 1.f / det;
    conic = make_float3(cov.z * det_inv, -cov.y * det_inv, cov.x * det_inv);
    const float mid = 0.5f * (cov.x + cov.z);
    const float lambda1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float lambda2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
    my_radius = ceilf(3.f * sqrtf(fmaxf(lambda1, lambda2)));
  }
  const float2 point_image = {ndc_to_pixel(scr_x, W), ndc_to_pixel(scr_y, H)};
  const int radius = (int)my_radius;
  int2 rmin, rmax;
  if (seam_wrap)
    tile_rect_cyclic(point_image, radius, gx, gy, rmin, rmax);
  else
    tile_rect(point_image, radius, gx, gy, rmin, rmax);
  const uint32_t area = (uint32_t)(rmax.x - rmin.x) * (uint32_t)(rmax.y - rmin.y);
  if (area == 0) return res;
  if (color_precomp == nullptr) {
    const V3 pos = v3(p_orig.x, p_orig.y, p_orig.z);
    const V3 cam = v3(campos[0], campos[1], campos[2]);
    const V3 c = sh_color_unclamped(D, pos, cam, sh);
    const uint32_t bits = (c.x < 0 ? 1u : 0u) | (c.y < 0 ? 2u : 0u) | (c.z < 0 ? 4u : 0u);
    res.col = make_float4(clamp_at_zero(c.x), clamp_at_zero(c.y), clamp_at_zero(c.z), __uint_as_float(bits));
  } else {
    res.col = make_float4(color_precomp[0], color_precomp[1], color_precomp[2], __uint_as_float(0u));
  }
  const float2 cull = cull_quadric(point_image.x, point_image.y, conic.x, conic.y, conic.z, opacity);
  res.s0 = make_float4(point_image.x, point_image.y, conic.x, conic.y);
  res.s1 = make_float4(conic.z, opacity, cull.x, cull.y);
  res.depth_key = r;
  res.radius = radius;
  res.touched = area;
  return res;
}

}  // namespace omnigs
