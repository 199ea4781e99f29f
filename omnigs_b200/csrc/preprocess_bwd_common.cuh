// Per-(view, Gaussian) pieces of the backward lonlat preprocess, shared by the single-view kernel
// and the batched multi-view kernel.  The FP32 expressions follow the reference's order
// (backward.cu:30-151, 297-485, 489-552, 613-669).
#pragma once

#include "device_util.cuh"
#include "lonlat_math.cuh"

namespace omnigs {

__device__ __forceinline__ V3 operator*(V3 v, float s) { return V3{v.x * s, v.y * s, v.z * s}; }
__device__ __forceinline__ float tsqrt(float v) { return sqrtf(v); }
__device__ __forceinline__ double tsqrt(double v) { return sqrt(v); }

// dnormvdv, auxiliary.h:134-144.
__device__ __forceinline__ float3 dnormvdv3(float3 v, float3 dv) {
  const float sum2 = v.x * v.x + v.y * v.y + v.z * v.z;
  const float invsum32 = 1.0f / sqrtf(sum2 * sum2 * sum2);
  float3 r;
  r.x = ((+sum2 - v.x * v.x) * dv.x - v.y * v.x * dv.y - v.z * v.x * dv.z) * invsum32;
  r.y = (-v.x * v.y * dv.x + (sum2 - v.y * v.y) * dv.y - v.z * v.y * dv.z) * invsum32;
  r.z = (-v.x * v.z * dv.x - v.y * v.z * dv.y + (sum2 - v.z * v.z) * dv.z) * invsum32;
  return r;
}

// computeCov2DLonLatCUDA (backward.cu:297-485) in scalar type T: from dL/dconic, writes dL/dcov3D
// (dcov, 6 values) and returns the covariance path's dL/dmean3D; `jac` receives the Jacobian rows
// dpx_dt / dpy_dt that the screen-space mean path needs.  T = float is the reference's arithmetic;
// T = double is the precision mode near the poles, where the Jacobian's 1/rho terms make the FP32
// inverse ill-conditioned.
template <class T>
__device__ __forceinline__ V3 cov2d_lonlat_backward(const float3& mean, const float* cov3D, const float* vm,
                                                    int W, int H, float3 dconic, float dcov[6],
                                                    LonlatJacobian& jac) {
  const T eps = T(0.0000001f);
  const T tx_ = T(vm[0]) * T(mean.x) + T(vm[4]) * T(mean.y) + T(vm[8]) * T(mean.z) + T(vm[12]);
  const T ty_ = T(vm[1]) * T(mean.x) + T(vm[5]) * T(mean.y) + T(vm[9]) * T(mean.z) + T(vm[13]);
  const T tz_ = T(vm[2]) * T(mean.x) + T(vm[6]) * T(mean.y) + T(vm[10]) * T(mean.z) + T(vm[14]);
  const T txtx = tx_ * tx_;
  const T tyty = ty_ * ty_;
  const T tztz = tz_ * tz_;
  const T txtytz = tx_ * ty_ * tz_;
  const T trxztrxz = txtx + tztz;
  const T trxztrxz_inv = T(1) / (trxztrxz + eps);
  const T trxztrxztrxztrxz_inv = trxztrxz_inv * trxztrxz_inv;
  const T trxz = tsqrt(trxztrxz);
  const T trxz_inv = T(1) / (trxz + eps);
  const T trtr = trxztrxz + tyty;
  const T trtr_inv = T(1) / (trtr + eps);
  const T trtrtrtr_inv = trtr_inv * trtr_inv;
  const T trxz_trtrtrtr_inv = trxz_inv * trtrtrtr_inv;
  const T trxztrxztrxz_trtrtrtr_inv = trxztrxz_inv * trxz_trtrtrtr_inv;
  const T tyty_minus_trxztrxz = tyty - trxztrxz;
  const T W_div_2pi = W * T(0.5f) * T(kInvPi);
  const T H_div_pi = H * T(kInvPi);
  const T dpx_dtx = W_div_2pi * tz_ * trxztrxz_inv;
  const T dpx_dtz = -W_div_2pi * tx_ * trxztrxz_inv;
  const T dpy_dtx = -H_div_pi * tx_ * ty_ * trxz_inv * trtr_inv;
  const T dpy_dty = H_div_pi * trxz * trtr_inv;
  const T dpy_dtz = -H_div_pi * tz_ * ty_ * trxz_inv * trtr_inv;
  jac.dpx_dtx = (float)dpx_dtx;
  jac.dpx_dtz = (float)dpx_dtz;
  jac.dpy_dtx = (float)dpy_dtx;
  jac.dpy_dty = (float)dpy_dty;
  jac.dpy_dtz = (float)dpy_dtz;

  const T zero = T(0);
  const Mat3<T> J = mat3_cols_t<T>(dpx_dtx, zero, dpx_dtz, dpy_dtx, dpy_dty, dpy_dtz, zero, zero, zero);
  const Mat3<T> Wm = mat3_cols_t<T>(vm[0], vm[4], vm[8], vm[1], vm[5], vm[9], vm[2], vm[6], vm[10]);
  const Mat3<T> Vrk = mat3_cols_t<T>(cov3D[0], cov3D[1], cov3D[2], cov3D[1], cov3D[3], cov3D[4], cov3D[2],
                                     cov3D[4], cov3D[5]);
  const Mat3<T> Tm3 = mat3_mul(Wm, J);
  Mat3<T> cov2D = mat3_mul(mat3_mul(mat3_transpose(Tm3), mat3_transpose(Vrk)), Tm3);
  const T a = cov2D.m[0][0] += T(0.3f);
  const T b = cov2D.m[0][1];
  const T c = cov2D.m[1][1] += T(0.3f);
  const T denom = a * c - b * b;
  T dL_da = 0, dL_db = 0, dL_dc = 0;
  const T denom2inv = T(1) / ((denom * denom) + eps);
  const T dcx = dconic.x, dcy = dconic.y, dcz = dconic.z;
  const auto& Tm = Tm3.m;
  T dc[6] = {0, 0, 0, 0, 0, 0};
  if (denom2inv != 0) {
    dL_da = denom2inv * (-c * c * dcx + 2 * b * c * dcy + (denom - a * c) * dcz);
    dL_dc = denom2inv * (-a * a * dcz + 2 * a * b * dcy + (denom - a * c) * dcx);
    dL_db = denom2inv * 2 * (b * c * dcx - (denom + 2 * b * b) * dcy + a * b * dcz);
    dc[0] = (Tm[0][0] * Tm[0][0] * dL_da + Tm[0][0] * Tm[1][0] * dL_db + Tm[1][0] * Tm[1][0] * dL_dc);
    dc[3] = (Tm[0][1] * Tm[0][1] * dL_da + Tm[0][1] * Tm[1][1] * dL_db + Tm[1][1] * Tm[1][1] * dL_dc);
    dc[5] = (Tm[0][2] * Tm[0][2] * dL_da + Tm[0][2] * Tm[1][2] * dL_db + Tm[1][2] * Tm[1][2] * dL_dc);
    dc[1] = 2 * Tm[0][0] * Tm[0][1] * dL_da + (Tm[0][0] * Tm[1][1] + Tm[0][1] * Tm[1][0]) * dL_db +
            2 * Tm[1][0] * Tm[1][1] * dL_dc;
    dc[2] = 2 * Tm[0][0] * Tm[0][2] * dL_da + (Tm[0][0] * Tm[1][2] + Tm[0][2] * Tm[1][0]) * dL_db +
            2 * Tm[1][0] * Tm[1][2] * dL_dc;
    dc[4] = 2 * Tm[0][2] * Tm[0][1] * dL_da + (Tm[0][1] * Tm[1][2] + Tm[0][2] * Tm[1][1]) * dL_db +
            2 * Tm[1][1] * Tm[1][2] * dL_dc;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) dcov[k] = (float)dc[k];

  const auto& V = Vrk.m;
  const T dL_dT00 = 2 * (Tm[0][0] * V[0][0] + Tm[0][1] * V[0][1] + Tm[0][2] * V[0][2]) * dL_da +
                    (Tm[1][0] * V[0][0] + Tm[1][1] * V[0][1] + Tm[1][2] * V[0][2]) * dL_db;
  const T dL_dT01 = 2 * (Tm[0][0] * V[1][0] + Tm[0][1] * V[1][1] + Tm[0][2] * V[1][2]) * dL_da +
                    (Tm[1][0] * V[1][0] + Tm[1][1] * V[1][1] + Tm[1][2] * V[1][2]) * dL_db;
  const T dL_dT02 = 2 * (Tm[0][0] * V[2][0] + Tm[0][1] * V[2][1] + Tm[0][2] * V[2][2]) * dL_da +
                    (Tm[1][0] * V[2][0] + Tm[1][1] * V[2][1] + Tm[1][2] * V[2][2]) * dL_db;
  const T dL_dT10 = 2 * (Tm[1][0] * V[0][0] + Tm[1][1] * V[0][1] + Tm[1][2] * V[0][2]) * dL_dc +
                    (Tm[0][0] * V[0][0] + Tm[0][1] * V[0][1] + Tm[0][2] * V[0][2]) * dL_db;
  const T dL_dT11 = 2 * (Tm[1][0] * V[1][0] + Tm[1][1] * V[1][1] + Tm[1][2] * V[1][2]) * dL_dc +
                    (Tm[0][0] * V[1][0] + Tm[0][1] * V[1][1] + Tm[0][2] * V[1][2]) * dL_db;
  const T dL_dT12 = 2 * (Tm[1][0] * V[2][0] + Tm[1][1] * V[2][1] + Tm[1][2] * V[2][2]) * dL_dc +
                    (Tm[0][0] * V[2][0] + Tm[0][1] * V[2][1] + Tm[0][2] * V[2][2]) * dL_db;
  const auto& Wg = Wm.m;
  const T dL_dJ00 = Wg[0][0] * dL_dT00 + Wg[0][1] * dL_dT01 + Wg[0][2] * dL_dT02;
  const T dL_dJ02 = Wg[2][0] * dL_dT00 + Wg[2][1] * dL_dT01 + Wg[2][2] * dL_dT02;
  const T dL_dJ10 = Wg[0][0] * dL_dT10 + Wg[0][1] * dL_dT11 + Wg[0][2] * dL_dT12;
  const T dL_dJ11 = Wg[1][0] * dL_dT10 + Wg[1][1] * dL_dT11 + Wg[1][2] * dL_dT12;
  const T dL_dJ12 = Wg[2][0] * dL_dT10 + Wg[2][1] * dL_dT11 + Wg[2][2] * dL_dT12;
  // second derivatives of the lonlat map (backward.cu:455-475; supp.pdf eqs. 43ff)
  const T temp1 = H_div_pi * tyty_minus_trxztrxz * trxz_trtrtrtr_inv;
  const T temp2 = H_div_pi * txtytz * (trtr + T(2) * trxztrxz) * trxztrxztrxz_trtrtrtr_inv;
  const T temp3 = W_div_2pi * (txtx - tztz) * trxztrxztrxztrxz_inv;
  const T temp4 = W_div_2pi * T(2) * tx_ * tz_ * trxztrxztrxztrxz_inv;
  const T temp5 = H_div_pi * ty_ * trxztrxztrxz_trtrtrtr_inv;
  const T dL_dtx = -dL_dJ00 * temp4 + dL_dJ02 * temp3 +
                   dL_dJ10 * temp5 * (T(2) * txtx * trxztrxz - tztz * trtr) + dL_dJ11 * tx_ * temp1 +
                   dL_dJ12 * temp2;
  const T dL_dty = dL_dJ10 * tx_ * temp1 - dL_dJ11 * H_div_pi * T(2) * trxz * ty_ * trtrtrtr_inv +
                   dL_dJ12 * tz_ * temp1;
  const T dL_dtz = dL_dJ00 * temp3 + dL_dJ02 * temp4 + dL_dJ10 * temp2 + dL_dJ11 * tz_ * temp1 +
                   dL_dJ12 * temp5 * (T(2) * tztz * trxztrxz - txtx * trtr);
  // W^T dL/dt (auxiliary.h transformVec4x3Transpose)
  const T mx = T(vm[0]) * dL_dtx + T(vm[1]) * dL_dty + T(vm[2]) * dL_dtz;
  const T my = T(vm[4]) * dL_dtx + T(vm[5]) * dL_dty + T(vm[6]) * dL_dtz;
  const T mz = T(vm[8]) * dL_dtx + T(vm[9]) * dL_dty + T(vm[10]) * dL_dtz;
  return v3((float)mx, (float)my, (float)mz);
}

// Screen-space mean path of preprocessLonLatCUDA (backward.cu:640-660): dL/dmean3D from the
// viewspace-point gradient (NDC scale) through the Jacobian rows.
__device__ __forceinline__ V3 mean2d_backward(const LonlatJacobian& j, float dmean2D_x, float dmean2D_y, int W,
                                              int H, const float* vm) {
  const float dsx_dpx = 2.0f / (float)W;
  const float dsy_dpy = 2.0f / (float)H;
  const float dL_dpx = dmean2D_x * dsx_dpx;
  const float dL_dpy = dmean2D_y * dsy_dpy;
  const float dtx = dL_dpx * j.dpx_dtx + dL_dpy * j.dpy_dtx;
  const float dty = dL_dpx * 0.0f + dL_dpy * j.dpy_dty;
  const float dtz = dL_dpx * j.dpx_dtz + dL_dpy * j.dpy_dtz;
  const float3 dm = xform_vec_T(float3{dtx, dty, dtz}, vm);
  return v3(dm.x, dm.y, dm.z);
}

// computeColorFromSH backward (backward.cu:30-151).  put(k, g) receives dL/dsh[k] for
// k < (deg + 1)^2; returns the view-direction term of dL/dmean3D.
template <class ShLoad, class Put>
__device__ __forceinline__ V3 sh_backward(int deg, V3 pos, V3 campos, ShLoad sh, uint32_t clamp_bits,
                                          V3 dL_dcolor, Put put) {
  const V3 dir_orig = pos - campos;
  const V3 dir = dir_orig / sqrtf(dot3(dir_orig, dir_orig));
  V3 dL_dRGB = dL_dcolor;
  dL_dRGB.x *= (clamp_bits & 1u) ? 0 : 1;
  dL_dRGB.y *= (clamp_bits & 2u) ? 0 : 1;
  dL_dRGB.z *= (clamp_bits & 4u) ? 0 : 1;
  V3 dRGBdx = v3(0, 0, 0), dRGBdy = v3(0, 0, 0), dRGBdz = v3(0, 0, 0);
  const float x = dir.x, y = dir.y, z = dir.z;
  const float dRGBdsh0 = kShC0;
  put(0, dRGBdsh0 * dL_dRGB);
  if (deg > 0) {
    const float dRGBdsh1 = -kShC1 * y;
    const float dRGBdsh2 = kShC1 * z;
    const float dRGBdsh3 = -kShC1 * x;
    put(1, dRGBdsh1 * dL_dRGB);
    put(2, dRGBdsh2 * dL_dRGB);
    put(3, dRGBdsh3 * dL_dRGB);
    dRGBdx = -kShC1 * sh(3);
    dRGBdy = -kShC1 * sh(1);
    dRGBdz = kShC1 * sh(2);
    if (deg > 1) {
      const float xx = x * x, yy = y * y, zz = z * z;
      const float xy = x * y, yz = y * z, xz = x * z;
      const float dRGBdsh4 = kShC2_0 * xy;
      const float dRGBdsh5 = kShC2_1 * yz;
      const float dRGBdsh6 = kShC2_2 * (2.f * zz - xx - yy);
      const float dRGBdsh7 = kShC2_3 * xz;
      const float dRGBdsh8 = kShC2_4 * (xx - yy);
      put(4, dRGBdsh4 * dL_dRGB);
      put(5, dRGBdsh5 * dL_dRGB);
      put(6, dRGBdsh6 * dL_dRGB);
      put(7, dRGBdsh7 * dL_dRGB);
      put(8, dRGBdsh8 * dL_dRGB);
      dRGBdx = dRGBdx + (kShC2_0 * y * sh(4) + kShC2_2 * 2.f * -x * sh(6) + kShC2_3 * z * sh(7) +
                         kShC2_4 * 2.f * x * sh(8));
      dRGBdy = dRGBdy + (kShC2_0 * x * sh(4) + kShC2_1 * z * sh(5) + kShC2_2 * 2.f * -y * sh(6) +
                         kShC2_4 * 2.f * -y * sh(8));
      dRGBdz = dRGBdz + (kShC2_1 * y * sh(5) + kShC2_2 * 2.f * 2.f * z * sh(6) + kShC2_3 * x * sh(7));
      if (deg > 2) {
        const float dRGBdsh9 = kShC3_0 * y * (3.f * xx - yy);
        const float dRGBdsh10 = kShC3_1 * xy * z;
        const float dRGBdsh11 = kShC3_2 * y * (4.f * zz - xx - yy);
        const float dRGBdsh12 = kShC3_3 * z * (2.f * zz - 3.f * xx - 3.f * yy);
        const float dRGBdsh13 = kShC3_4 * x * (4.f * zz - xx - yy);
        const float dRGBdsh14 = kShC3_5 * z * (xx - yy);
        const float dRGBdsh15 = kShC3_6 * x * (xx - 3.f * yy);
        put(9, dRGBdsh9 * dL_dRGB);
        put(10, dRGBdsh10 * dL_dRGB);
        put(11, dRGBdsh11 * dL_dRGB);
        put(12, dRGBdsh12 * dL_dRGB);
        put(13, dRGBdsh13 * dL_dRGB);
        put(14, dRGBdsh14 * dL_dRGB);
        put(15, dRGBdsh15 * dL_dRGB);
        dRGBdx = dRGBdx + (kShC3_0 * sh(9) * 3.f * 2.f * xy + kShC3_1 * sh(10) * yz +
                           kShC3_2 * sh(11) * -2.f * xy + kShC3_3 * sh(12) * -3.f * 2.f * xz +
                           kShC3_4 * sh(13) * (-3.f * xx + 4.f * zz - yy) + kShC3_5 * sh(14) * 2.f * xz +
                           kShC3_6 * sh(15) * 3.f * (xx - yy));
        dRGBdy = dRGBdy + (kShC3_0 * sh(9) * 3.f * (xx - yy) + kShC3_1 * sh(10) * xz +
                           kShC3_2 * sh(11) * (-3.f * yy + 4.f * zz - xx) + kShC3_3 * sh(12) * -3.f * 2.f * yz +
                           kShC3_4 * sh(13) * -2.f * xy + kShC3_5 * sh(14) * -2.f * yz +
                           kShC3_6 * sh(15) * -3.f * 2.f * xy);
        dRGBdz = dRGBdz + (kShC3_1 * sh(10) * xy + kShC3_2 * sh(11) * 4.f * 2.f * yz +
                           kShC3_3 * sh(12) * 3.f * (2.f * zz - xx - yy) + kShC3_4 * sh(13) * 4.f * 2.f * xz +
                           kShC3_5 * sh(14) * (xx - yy));
      }
    }
  }
  const V3 dL_ddir = v3(dot3(dRGBdx, dL_dRGB), dot3(dRGBdy, dL_dRGB), dot3(dRGBdz, dL_dRGB));
  const float3 dn = dnormvdv3(float3{dir_orig.x, dir_orig.y, dir_orig.z}, float3{dL_ddir.x, dL_ddir.y, dL_ddir.z});
  return v3(dn.x, dn.y, dn.z);
}

// computeCov3D backward (backward.cu:489-552): dL/dscale and dL/drot from dL/dcov3D (linear in
// dcov, so a batch may sum dcov over its views first).  No gradient through the quaternion
// normalisation, as in the reference (backward.cu:551).
__device__ __forceinline__ void cov3d_backward(float3 scale, float mod, float4 q, const float* d, float dscale[3],
                                               float drot[4]) {
  const float r = q.x, x = q.y, y = q.z, z = q.w;
  const Mat3c R = mat3_cols(1.f - 2.f * (y * y + z * z), 2.f * (x * y - r * z), 2.f * (x * z + r * y),
                            2.f * (x * y + r * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - r * x),
                            2.f * (x * z - r * y), 2.f * (y * z + r * x), 1.f - 2.f * (x * x + y * y));
  Mat3c S = mat3_identity();
  const V3 s = mod * v3(scale.x, scale.y, scale.z);
  S.m[0][0] = s.x;
  S.m[1][1] = s.y;
  S.m[2][2] = s.z;
  const Mat3c Mm = mat3_mul(S, R);
  const Mat3c dL_dSigma = mat3_cols(d[0], 0.5f * d[1], 0.5f * d[2], 0.5f * d[1], d[3], 0.5f * d[4],
                                    0.5f * d[2], 0.5f * d[4], d[5]);
  Mat3c twoM;
  for (int cc = 0; cc < 3; ++cc)
    for (int rr = 0; rr < 3; ++rr) twoM.m[cc][rr] = Mm.m[cc][rr] * 2.0f;
  const Mat3c dL_dM = mat3_mul(twoM, dL_dSigma);
  const Mat3c Rt = mat3_transpose(R);
  Mat3c dL_dMt = mat3_transpose(dL_dM);
  dscale[0] = Rt.m[0][0] * dL_dMt.m[0][0] + Rt.m[0][1] * dL_dMt.m[0][1] + Rt.m[0][2] * dL_dMt.m[0][2];
  dscale[1] = Rt.m[1][0] * dL_dMt.m[1][0] + Rt.m[1][1] * dL_dMt.m[1][1] + Rt.m[1][2] * dL_dMt.m[1][2];
  dscale[2] = Rt.m[2][0] * dL_dMt.m[2][0] + Rt.m[2][1] * dL_dMt.m[2][1] + Rt.m[2][2] * dL_dMt.m[2][2];
  for (int rr = 0; rr < 3; ++rr) {
    dL_dMt.m[0][rr] *= s.x;
    dL_dMt.m[1][rr] *= s.y;
    dL_dMt.m[2][rr] *= s.z;
  }
  const auto& G = dL_dMt.m;
  drot[0] = 2 * z * (G[0][1] - G[1][0]) + 2 * y * (G[2][0] - G[0][2]) + 2 * x * (G[1][2] - G[2][1]);
  drot[1] = 2 * y * (G[1][0] + G[0][1]) + 2 * z * (G[2][0] + G[0][2]) + 2 * r * (G[1][2] - G[2][1]) -
            4 * x * (G[2][2] + G[1][1]);
  drot[2] = 2 * x * (G[1][0] + G[0][1]) + 2 * r * (G[2][0] - G[0][2]) + 2 * z * (G[1][2] + G[2][1]) -
            4 * y * (G[2][2] + G[0][0]);
  drot[3] = 2 * r * (G[0][1] - G[1][0]) + 2 * x * (G[2][0] + G[0][2]) + 2 * y * (G[1][2] + G[2][1]) -
            4 * z * (G[1][1] + G[0][0]);
}

}  // namespace omnigs
