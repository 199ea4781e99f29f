// Per-Gaussian lonlat (equirectangular) math, FP32.
//
// The integer outputs of the preprocess (radii, tile rects, tiles_touched) and everything keyed
// on them (the sorted instance list, the tile ranges) must be bit-exact with the reference
// rasterizer.  They depend on the exact FP32 operation sequence, including which products the
// compiler fuses into FMAs, so the functions here evaluate the same expression trees as
// cuda_rasterizer/forward.cu and auxiliary.h.  Mat3c is a column-major 3x3 matrix whose product
// is evaluated term by term in the same order as the reference's glm::mat3 product
// (r[c][i] = a[0][i] b[c][0] + a[1][i] b[c][1] + a[2][i] b[c][2]); nothing here may be built with
// --use_fast_math.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace omnigs {

constexpr int kTileW = 16;  // cuda_rasterizer/config.h:26-27 (BLOCK_X, BLOCK_Y)
constexpr int kTileH = 16;

// Real spherical-harmonics basis constants (values of auxiliary.h:32-49).
constexpr float kShC0 = 0.28209479177387814f;
constexpr float kShC1 = 0.4886025119029199f;
constexpr float kShC2_0 = 1.0925484305920792f;
constexpr float kShC2_1 = -1.0925484305920792f;
constexpr float kShC2_2 = 0.31539156525252005f;
constexpr float kShC2_3 = -1.0925484305920792f;
constexpr float kShC2_4 = 0.5462742152960396f;
constexpr float kShC3_0 = -0.5900435899266435f;
constexpr float kShC3_1 = 2.890611442640554f;
constexpr float kShC3_2 = -0.4570457994644658f;
constexpr float kShC3_3 = 0.3731763325901154f;
constexpr float kShC3_4 = -0.4570457994644658f;
constexpr float kShC3_5 = 1.445305721320277f;
constexpr float kShC3_6 = -0.5900435899266435f;

constexpr float kInvPi = 0.318309886183790671537767526745028724f;  // M_1_PIf32
constexpr float kTwoInvPi = 0.636619772367581343075535053490057448f;  // M_2_PIf32

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(float s, V3 v) { return V3{s * v.x, s * v.y, s * v.z}; }
__device__ __forceinline__ V3 operator/(V3 v, float s) { return V3{v.x / s, v.y / s, v.z / s}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

template <class T>
struct Mat3 {
  T m[3][3];  // m[column][row]
};
using Mat3c = Mat3<float>;
template <class T>
__device__ __forceinline__ Mat3<T> mat3_cols_t(T a0, T a1, T a2, T a3, T a4, T a5, T a6, T a7, T a8) {
  Mat3<T> r;
  r.m[0][0] = a0; r.m[0][1] = a1; r.m[0][2] = a2;
  r.m[1][0] = a3; r.m[1][1] = a4; r.m[1][2] = a5;
  r.m[2][0] = a6; r.m[2][1] = a7; r.m[2][2] = a8;
  return r;
}
__device__ __forceinline__ Mat3c mat3_cols(float a0, float a1, float a2, float a3, float a4, float a5,
                                           float a6, float a7, float a8) {
  return mat3_cols_t<float>(a0, a1, a2, a3, a4, a5, a6, a7, a8);
}
__device__ __forceinline__ Mat3c mat3_identity() { return mat3_cols(1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f); }
template <class T>
__device__ __forceinline__ Mat3<T> mat3_mul(const Mat3<T>& a, const Mat3<T>& b) {
  Mat3<T> r;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      r.m[c][i] = a.m[0][i] * b.m[c][0] + a.m[1][i] * b.m[c][1] + a.m[2][i] * b.m[c][2];
  return r;
}
template <class T>
__device__ __forceinline__ Mat3<T> mat3_transpose(const Mat3<T>& a) {
  Mat3<T> r;
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int i = 0; i < 3; ++i) r.m[c][i] = a.m[i][c];
  return r;
}

// Tcw applied to a point / transposed rotation applied to a vector (auxiliary.h:85-124); the
// matrix is the row-major storage of Tcw^T, i.e. Tcw column-major.
__device__ __forceinline__ float3 xform_point(const float3& p, const float* m) {
  return float3{m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
                m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
                m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]};
}
__device__ __forceinline__ float3 xform_vec_T(const float3& p, const float* m) {
  return float3{m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z,
                m[8] * p.x + m[9] * p.y + m[10] * p.z};
}
__device__ __forceinline__ Mat3c view_rotation(const float* v) {  // forward.cu:169-172
  return mat3_cols(v[0], v[4], v[8], v[1], v[5], v[9], v[2], v[6], v[10]);
}

// ndc2Pix, auxiliary.h:51-54: the literals are doubles, so the map is evaluated in FP64.
__device__ __forceinline__ float ndc_to_pixel(float v, int S) { return ((v + 1.0) * S - 1.0) * 0.5; }

// Clamped tile rectangle of a splat (getRect, auxiliary.h:56-66).  The lonlat path uses this
// clamp, not the cyclic variant (forward.cu:680-681, rasterizer_impl.cu:117).
__device__ __forceinline__ void tile_rect(float2 p, int max_radius, int gx, int gy, int2& rmin,
                                          int2& rmax) {
  rmin.x = min(gx, max(0, (int)((p.x - max_radius) / kTileW)));
  rmin.y = min(gy, max(0, (int)((p.y - max_radius) / kTileH)));
  rmax.x = min(gx, max(0, (int)((p.x + max_radius + kTileW - 1) / kTileW)));
  rmax.y = min(gy, max(0, (int)((p.y + max_radius + kTileH - 1) / kTileH)));
}

// Seam-wrapping variant (the reference's unused getRectCyclic, auxiliary.h:68-83): the tile-column
// range may start left of column 0 (down to -gx) and end right of gx (up to 2 gx); the caller wraps
// column indices modulo gx.  Unlike getRectCyclic the left edge is floored, so a splat reaching
// less than a tile past x = 0 still gets the wrapped column, and the range is capped at one image
// width so no column is listed twice.  Rows are clamped as in getRect.
__device__ __forceinline__ void tile_rect_cyclic(float2 p, int max_radius, int gx, int gy, int2& rmin, int2& rmax) {
  rmin.x = min(gx, max(-gx, (int)floorf((p.x - max_radius) / kTileW)));
  rmin.y = min(gy, max(0, (int)((p.y - max_radius) / kTileH)));
  rmax.x = min(2 * gx, max(0, (int)((p.x + max_radius + kTileW - 1) / kTileW)));
  rmax.y = min(gy, max(0, (int)((p.y + max_radius + kTileH - 1) / kTileH)));
  if (rmax.x < rmin.x) rmax.x = rmin.x;
  if (rmax.x - rmin.x > gx) rmax.x = rmin.x + gx;
}

// 3D covariance from scale and (unnormalised) quaternion (r, x, y, z), forward.cu:194-228.
__device__ __forceinline__ void cov3d_from_scale_rot(float3 s, float mod, float4 q, float out[6]) {
  Mat3c S = mat3_identity();
  S.m[0][0] = mod * s.x;
  S.m[1][1] = mod * s.y;
  S.m[2][2] = mod * s.z;
  const float r = q.x, x = q.y, y = q.z, z = q.w;
  Mat3c R = mat3_cols(1.f - 2.f * (y * y + z * z), 2.f * (x * y - r * z), 2.f * (x * z + r * y),
                      2.f * (x * y + r * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - r * x),
                      2.f * (x * z - r * y), 2.f * (y * z + r * x), 1.f - 2.f * (x * x + y * y));
  Mat3c M = mat3_mul(S, R);
  Mat3c Sig = mat3_mul(mat3_transpose(M), M);
  out[0] = Sig.m[0][0];
  out[1] = Sig.m[0][1];
  out[2] = Sig.m[0][2];
  out[3] = Sig.m[1][1];
  out[4] = Sig.m[1][2];
  out[5] = Sig.m[2][2];
}

// The equirectangular Jacobian d(px, py)/dt, forward.cu:147-162 (the same sequence is recomputed
// by the backward, backward.cu:340-360).
struct LonlatJacobian {
  float dpx_dtx, dpx_dtz, dpy_dtx, dpy_dty, dpy_dtz;
};
__device__ __forceinline__ LonlatJacobian lonlat_jacobian(float3 t, int width, int height) {
  const float trxztrxz = t.x * t.x + t.z * t.z;
  const float trxztrxz_inv = 1.0f / (trxztrxz + 0.0000001f);
  const float trxz = sqrtf(trxztrxz);
  const float trxz_inv = 1.0f / (trxz + 0.0000001f);
  const float trtr = trxztrxz + t.y * t.y;
  const float trtr_inv = 1.0f / (trtr + 0.0000001f);
  const float W_div_2pi = width * 0.5f * kInvPi;
  const float H_div_pi = height * kInvPi;
  LonlatJacobian j;
  j.dpx_dtx = W_div_2pi * t.z * trxztrxz_inv;
  j.dpx_dtz = -W_div_2pi * t.x * trxztrxz_inv;
  j.dpy_dtx = -H_div_pi * t.x * t.y * trxz_inv * trtr_inv;
  j.dpy_dty = H_div_pi * trxz * trtr_inv;
  j.dpy_dtz = -H_div_pi * t.z * t.y * trxz_inv * trtr_inv;
  return j;
}

// EWA screen-space covariance of a lonlat splat plus the 0.3 px^2 low-pass (forward.cu:130-189).
__device__ __forceinline__ float3 cov2d_lonlat(const float3& mean, int width, int height,
                                               const float* cov3D, const float* viewmatrix) {
  const float3 t = xform_point(mean, viewmatrix);
  const LonlatJacobian j = lonlat_jacobian(t, width, height);
  Mat3c J = mat3_cols(j.dpx_dtx, 0.0f, j.dpx_dtz, j.dpy_dtx, j.dpy_dty, j.dpy_dtz, 0.0f, 0.0f, 0.0f);
  Mat3c W = view_rotation(viewmatrix);
  Mat3c T = mat3_mul(W, J);
  Mat3c Vrk = mat3_cols(cov3D[0], cov3D[1], cov3D[2], cov3D[1], cov3D[3], cov3D[4], cov3D[2],
                        cov3D[4], cov3D[5]);
  Mat3c cov = mat3_mul(mat3_mul(mat3_transpose(T), mat3_transpose(Vrk)), T);
  cov.m[0][0] += 0.3f;
  cov.m[1][1] += 0.3f;
  return float3{cov.m[0][0], cov.m[0][1], cov.m[1][1]};
}

// Gradients of the pixel coordinates with respect to the world-space mean, in FP64: column c of
// the reference's T = W J (forward.cu:164-176), i.e. g[c][i] = sum_k R^T(i, k) d(p_c)/d(t_k), with
// the same 1e-7 guards as the FP32 Jacobian.  Used by the precision mode near the poles.
struct LonlatGradF64 {
  double gx[3], gy[3];
};
__device__ __forceinline__ LonlatGradF64 lonlat_grad_f64(const float3& mean, int width, int height,
                                                         const float* vm) {
  const double tx = (double)vm[0] * mean.x + (double)vm[4] * mean.y + (double)vm[8] * mean.z + vm[12];
  const double ty = (double)vm[1] * mean.x + (double)vm[5] * mean.y + (double)vm[9] * mean.z + vm[13];
  const double tz = (double)vm[2] * mean.x + (double)vm[6] * mean.y + (double)vm[10] * mean.z + vm[14];
  const double rxz2 = tx * tx + tz * tz;
  const double rxz2_inv = 1.0 / (rxz2 + 1e-7);
  const double rxz = sqrt(rxz2);
  const double rxz_inv = 1.0 / (rxz + 1e-7);
  const double rr = rxz2 + ty * ty;
  const double rr_inv = 1.0 / (rr + 1e-7);
  const double w2pi = width * 0.5 / 3.14159265358979323846;
  const double hpi = height / 3.14159265358979323846;
  const double jx[3] = {w2pi * tz * rxz2_inv, 0.0, -w2pi * tx * rxz2_inv};
  const double jy[3] = {-hpi * tx * ty * rxz_inv * rr_inv, hpi * rxz * rr_inv, -hpi * tz * ty * rxz_inv * rr_inv};
  LonlatGradF64 g;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    g.gx[i] = (double)vm[4 * i] * jx[0] + (double)vm[4 * i + 1] * jx[1] + (double)vm[4 * i + 2] * jx[2];
    g.gy[i] = (double)vm[4 * i] * jy[0] + (double)vm[4 * i + 1] * jy[1] + (double)vm[4 * i + 2] * jy[2];
  }
  return g;
}

// u^T Sigma v for the symmetric 3D covariance stored as (xx, xy, xz, yy, yz, zz).
__device__ __forceinline__ double sym_form_f64(const float* s, const double* u, const double* v) {
  const double su0 = s[0] * u[0] + s[1] * u[1] + s[2] * u[2];
  const double su1 = s[1] * u[0] + s[3] * u[1] + s[4] * u[2];
  const double su2 = s[2] * u[0] + s[4] * u[1] + s[5] * u[2];
  return su0 * v[0] + su1 * v[1] + su2 * v[2];
}

// cov2d_lonlat in FP64: (a, b, c) of the screen-space covariance including the 0.3 low-pass.
__device__ __forceinline__ double3 cov2d_lonlat_f64(const float3& mean, int width, int height,
                                                    const float* cov3D, const float* viewmatrix) {
  const LonlatGradF64 g = lonlat_grad_f64(mean, width, height, viewmatrix);
  return make_double3(sym_form_f64(cov3D, g.gx, g.gx) + 0.3, sym_form_f64(cov3D, g.gx, g.gy),
                      sym_form_f64(cov3D, g.gy, g.gy) + 0.3);
}

// View-dependent colour from degree-<=3 SH (forward.cu:30-83).  `sh` points at this Gaussian's
// coefficients (coefficient-major, RGB inner).  Returns the colour before clamping; the caller
// records the clamp flags and clamps at zero.
template <class ShLoad>
__device__ __forceinline__ V3 sh_color_unclamped(int deg, V3 pos, V3 campos, ShLoad sh) {
  V3 dir = pos - campos;
  dir = dir / sqrtf(dot3(dir, dir));
  V3 result = kShC0 * sh(0);
  if (deg > 0) {
    const float x = dir.x, y = dir.y, z = dir.z;
    result = result - kShC1 * y * sh(1) + kShC1 * z * sh(2) - kShC1 * x * sh(3);
    if (deg > 1) {
      const float xx = x * x, yy = y * y, zz = z * z;
      const float xy = x * y, yz = y * z, xz = x * z;
      result = result + kShC2_0 * xy * sh(4) + kShC2_1 * yz * sh(5) +
               kShC2_2 * (2.0f * zz - xx - yy) * sh(6) + kShC2_3 * xz * sh(7) +
               kShC2_4 * (xx - yy) * sh(8);
      if (deg > 2) {
        result = result + kShC3_0 * y * (3.0f * xx - yy) * sh(9) + kShC3_1 * xy * z * sh(10) +
                 kShC3_2 * y * (4.0f * zz - xx - yy) * sh(11) +
                 kShC3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * sh(12) +
                 kShC3_4 * x * (4.0f * zz - xx - yy) * sh(13) + kShC3_5 * z * (xx - yy) * sh(14) +
                 kShC3_6 * x * (xx - 3.0f * yy) * sh(15);
      }
    }
  }
  result.x += 0.5f;
  result.y += 0.5f;
  result.z += 0.5f;
  return result;
}

__device__ __forceinline__ float clamp_at_zero(float v) { return (v < 0.0f) ? 0.0f : v; }

}  // namespace omnigs
