// Backward of the lonlat preprocess, one thread per Gaussian, fused into one kernel.
//
// The reference runs two kernels and round-trips dL/dmeans3D and the Jacobian rows dpx_dt /
// dpy_dt through global memory (backward.cu:948-1016): computeCov2DLonLatCUDA (:297-485) then
// preprocessLonLatCUDA (:613-669) with the SH backward (:30-151) and the scale/rotation backward
// (:489-552).  Here one thread does all of it in registers, recomputes cov3D from scale and
// rotation (bit-identical to the forward) instead of reading a stored copy, consumes and clears the
// per-splat accumulator record written by the backward blend, and writes every output for every
// Gaussian (zeros for culled ones), so callers need not pre-zero anything.  The FP32 expressions
// follow the reference's order.
#include "device_util.cuh"
#include "kernels.h"
#include "lonlat_math.cuh"

namespace omnigs {
namespace {

__device__ __forceinline__ V3 operator*(V3 v, float s) { return V3{v.x * s, v.y * s, v.z * s}; }

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

__global__ void __launch_bounds__(256) preprocess_backward_kernel(PreprocessBackwardParams p) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= p.P) return;
  const int M = p.M;
  float* dsh = (p.dL_dsh != nullptr && M > 0) ? p.dL_dsh + (size_t)idx * M * 3 : nullptr;

  if (!(p.radii[idx] > 0)) {
    for (int k = 0; k < 3; ++k) {
      p.dL_dmeans2D[3 * idx + k] = 0.f;
      p.dL_dcolors[3 * idx + k] = 0.f;
      p.dL_dmeans3D[3 * idx + k] = 0.f;
      p.dL_dscales[3 * idx + k] = 0.f;
    }
    if (p.dL_dconic)
      for (int k = 0; k < 4; ++k) p.dL_dconic[4 * idx + k] = 0.f;
    p.dL_dopacity[idx] = 0.f;
    for (int k = 0; k < 6; ++k) p.dL_dcov3D[6 * idx + k] = 0.f;
    for (int k = 0; k < 4; ++k) p.dL_drotations[4 * idx + k] = 0.f;
    if (dsh)
      for (int k = 0; k < 3 * M; ++k) dsh[k] = 0.f;
    return;
  }

  // ---- consume the accumulator record of the backward blend ----
  const float4 g0 = p.grad_acc[3 * idx];
  const float4 g1 = p.grad_acc[3 * idx + 1];
  const float4 g2 = p.grad_acc[3 * idx + 2];
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  p.grad_acc[3 * idx] = z4;
  p.grad_acc[3 * idx + 1] = z4;
  p.grad_acc[3 * idx + 2] = z4;
  const float dmean2D_x = g0.x, dmean2D_y = g0.y;
  const float3 dL_dconic = {g0.z, g0.w, g1.x};
  const float dL_dcolor[3] = {g1.z, g1.w, g2.x};
  p.dL_dmeans2D[3 * idx] = dmean2D_x;
  p.dL_dmeans2D[3 * idx + 1] = dmean2D_y;
  p.dL_dmeans2D[3 * idx + 2] = 0.f;
  if (p.dL_dconic) {
    p.dL_dconic[4 * idx] = g0.z;
    p.dL_dconic[4 * idx + 1] = g0.w;
    p.dL_dconic[4 * idx + 2] = 0.f;
    p.dL_dconic[4 * idx + 3] = g1.x;
  }
  p.dL_dopacity[idx] = g1.y;
  p.dL_dcolors[3 * idx] = dL_dcolor[0];
  p.dL_dcolors[3 * idx + 1] = dL_dcolor[1];
  p.dL_dcolors[3 * idx + 2] = dL_dcolor[2];

  // ---- computeCov2DLonLatCUDA (backward.cu:297-485) ----
  const float* vm = p.viewmatrix;
  const float3 mean = {p.means3D[3 * idx], p.means3D[3 * idx + 1], p.means3D[3 * idx + 2]};
  float cov3D[6];
  if (p.cov3D_precomp != nullptr) {
    for (int k = 0; k < 6; ++k) cov3D[k] = p.cov3D_precomp[6 * idx + k];
  } else {
    const float3 s = {p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]};
    const float4 q = {p.rotations[4 * idx], p.rotations[4 * idx + 1], p.rotations[4 * idx + 2],
                      p.rotations[4 * idx + 3]};
    cov3d_from_scale_rot(s, p.scale_modifier, q, cov3D);
  }
  const float3 t = xform_point(mean, vm);
  const float txtx = t.x * t.x;
  const float tyty = t.y * t.y;
  const float tztz = t.z * t.z;
  const float txtytz = t.x * t.y * t.z;
  const float trxztrxz = txtx + tztz;
  const float trxztrxz_inv = 1.0f / (trxztrxz + 0.0000001f);
  const float trxztrxztrxztrxz_inv = trxztrxz_inv * trxztrxz_inv;
  const float trxz = sqrtf(trxztrxz);
  const float trxz_inv = 1.0f / (trxz + 0.0000001f);
  const float trtr = trxztrxz + tyty;
  const float trtr_inv = 1.0f / (trtr + 0.0000001f);
  const float trtrtrtr_inv = trtr_inv * trtr_inv;
  const float trxz_trtrtrtr_inv = trxz_inv * trtrtrtr_inv;
  const float trxztrxztrxz_trtrtrtr_inv = trxztrxz_inv * trxz_trtrtrtr_inv;
  const float tyty_minus_trxztrxz = tyty - trxztrxz;
  const float W_div_2pi = p.W * 0.5f * kInvPi;
  const float H_div_pi = p.H * kInvPi;
  const float dpx_dtx = W_div_2pi * t.z * trxztrxz_inv;
  const float dpx_dtz = -W_div_2pi * t.x * trxztrxz_inv;
  const float dpy_dtx = -H_div_pi * t.x * t.y * trxz_inv * trtr_inv;
  const float dpy_dty = H_div_pi * trxz * trtr_inv;
  const float dpy_dtz = -H_div_pi * t.z * t.y * trxz_inv * trtr_inv;

  const Mat3c J = mat3_cols(dpx_dtx, 0.0f, dpx_dtz, dpy_dtx, dpy_dty, dpy_dtz, 0.0f, 0.0f, 0.0f);
  const Mat3c Wm = view_rotation(vm);
  const Mat3c Vrk = mat3_cols(cov3D[0], cov3D[1], cov3D[2], cov3D[1], cov3D[3], cov3D[4], cov3D[2],
                              cov3D[4], cov3D[5]);
  const Mat3c T = mat3_mul(Wm, J);
  Mat3c cov2D = mat3_mul(mat3_mul(mat3_transpose(T), mat3_transpose(Vrk)), T);
  const float a = cov2D.m[0][0] += 0.3f;
  const float b = cov2D.m[0][1];
  const float c = cov2D.m[1][1] += 0.3f;
  const float denom = a * c - b * b;
  float dL_da = 0, dL_db = 0, dL_dc = 0;
  const float denom2inv = 1.0f / ((denom * denom) + 0.0000001f);
  float dcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const auto& Tm = T.m;
  if (denom2inv != 0) {
    dL_da = denom2inv * (-c * c * dL_dconic.x + 2 * b * c * dL_dconic.y + (denom - a * c) * dL_dconic.z);
    dL_dc = denom2inv * (-a * a * dL_dconic.z + 2 * a * b * dL_dconic.y + (denom - a * c) * dL_dconic.x);
    dL_db = denom2inv * 2 * (b * c * dL_dconic.x - (denom + 2 * b * b) * dL_dconic.y + a * b * dL_dconic.z);
    dcov[0] = (Tm[0][0] * Tm[0][0] * dL_da + Tm[0][0] * Tm[1][0] * dL_db + Tm[1][0] * Tm[1][0] * dL_dc);
    dcov[3] = (Tm[0][1] * Tm[0][1] * dL_da + Tm[0][1] * Tm[1][1] * dL_db + Tm[1][1] * Tm[1][1] * dL_dc);
    dcov[5] = (Tm[0][2] * Tm[0][2] * dL_da + Tm[0][2] * Tm[1][2] * dL_db + Tm[1][2] * Tm[1][2] * dL_dc);
    dcov[1] = 2 * Tm[0][0] * Tm[0][1] * dL_da + (Tm[0][0] * Tm[1][1] + Tm[0][1] * Tm[1][0]) * dL_db +
              2 * Tm[1][0] * Tm[1][1] * dL_dc;
    dcov[2] = 2 * Tm[0][0] * Tm[0][2] * dL_da + (Tm[0][0] * Tm[1][2] + Tm[0][2] * Tm[1][0]) * dL_db +
              2 * Tm[1][0] * Tm[1][2] * dL_dc;
    dcov[4] = 2 * Tm[0][2] * Tm[0][1] * dL_da + (Tm[0][1] * Tm[1][2] + Tm[0][2] * Tm[1][1]) * dL_db +
              2 * Tm[1][1] * Tm[1][2] * dL_dc;
  }
  for (int k = 0; k < 6; ++k) p.dL_dcov3D[6 * idx + k] = dcov[k];

  const auto& V = Vrk.m;
  const float dL_dT00 = 2 * (Tm[0][0] * V[0][0] + Tm[0][1] * V[0][1] + Tm[0][2] * V[0][2]) * dL_da +
                        (Tm[1][0] * V[0][0] + Tm[1][1] * V[0][1] + Tm[1][2] * V[0][2]) * dL_db;
  const float dL_dT01 = 2 * (Tm[0][0] * V[1][0] + Tm[0][1] * V[1][1] + Tm[0][2] * V[1][2]) * dL_da +
                        (Tm[1][0] * V[1][0] + Tm[1][1] * V[1][1] + Tm[1][2] * V[1][2]) * dL_db;
  const float dL_dT02 = 2 * (Tm[0][0] * V[2][0] + Tm[0][1] * V[2][1] + Tm[0][2] * V[2][2]) * dL_da +
                        (Tm[1][0] * V[2][0] + Tm[1][1] * V[2][1] + Tm[1][2] * V[2][2]) * dL_db;
  const float dL_dT10 = 2 * (Tm[1][0] * V[0][0] + Tm[1][1] * V[0][1] + Tm[1][2] * V[0][2]) * dL_dc +
                        (Tm[0][0] * V[0][0] + Tm[0][1] * V[0][1] + Tm[0][2] * V[0][2]) * dL_db;
  const float dL_dT11 = 2 * (Tm[1][0] * V[1][0] + Tm[1][1] * V[1][1] + Tm[1][2] * V[1][2]) * dL_dc +
                        (Tm[0][0] * V[1][0] + Tm[0][1] * V[1][1] + Tm[0][2] * V[1][2]) * dL_db;
  const float dL_dT12 = 2 * (Tm[1][0] * V[2][0] + Tm[1][1] * V[2][1] + Tm[1][2] * V[2][2]) * dL_dc +
                        (Tm[0][0] * V[2][0] + Tm[0][1] * V[2][1] + Tm[0][2] * V[2][2]) * dL_db;
  const auto& Wg = Wm.m;
  const float dL_dJ00 = Wg[0][0] * dL_dT00 + Wg[0][1] * dL_dT01 + Wg[0][2] * dL_dT02;
  const float dL_dJ02 = Wg[2][0] * dL_dT00 + Wg[2][1] * dL_dT01 + Wg[2][2] * dL_dT02;
  const float dL_dJ10 = Wg[0][0] * dL_dT10 + Wg[0][1] * dL_dT11 + Wg[0][2] * dL_dT12;
  const float dL_dJ11 = Wg[1][0] * dL_dT10 + Wg[1][1] * dL_dT11 + Wg[1][2] * dL_dT12;
  const float dL_dJ12 = Wg[2][0] * dL_dT10 + Wg[2][1] * dL_dT11 + Wg[2][2] * dL_dT12;
  // second derivatives of the lonlat map (backward.cu:455-475; supp.pdf eqs. 43ff)
  const float temp1 = H_div_pi * tyty_minus_trxztrxz * trxz_trtrtrtr_inv;
  const float temp2 = H_div_pi * txtytz * (trtr + 2.0f * trxztrxz) * trxztrxztrxz_trtrtrtr_inv;
  const float temp3 = W_div_2pi * (txtx - tztz) * trxztrxztrxztrxz_inv;
  const float temp4 = W_div_2pi * 2.0f * t.x * t.z * trxztrxztrxztrxz_inv;
  const float temp5 = H_div_pi * t.y * trxztrxztrxz_trtrtrtr_inv;
  const float dL_dtx = -dL_dJ00 * temp4 + dL_dJ02 * temp3 +
                       dL_dJ10 * temp5 * (2.0f * txtx * trxztrxz - tztz * trtr) + dL_dJ11 * t.x * temp1 +
                       dL_dJ12 * temp2;
  const float dL_dty = dL_dJ10 * t.x * temp1 - dL_dJ11 * H_div_pi * 2.0f * trxz * t.y * trtrtrtr_inv +
                       dL_dJ12 * t.z * temp1;
  const float dL_dtz = dL_dJ00 * temp3 + dL_dJ02 * temp4 + dL_dJ10 * temp2 + dL_dJ11 * t.z * temp1 +
                       dL_dJ12 * temp5 * (2.0f * tztz * trxztrxz - txtx * trtr);
  const float3 dm_cov = xform_vec_T(float3{dL_dtx, dL_dty, dL_dtz}, vm);
  V3 dL_dmeans = v3(dm_cov.x, dm_cov.y, dm_cov.z);

  // ---- preprocessLonLatCUDA: screen-space mean path (backward.cu:640-660) ----
  {
    const float dsx_dpx = 2.0f / (float)p.W;
    const float dsy_dpy = 2.0f / (float)p.H;
    const float dL_dpx = dmean2D_x * dsx_dpx;
    const float dL_dpy = dmean2D_y * dsy_dpy;
    const float dtx = dL_dpx * dpx_dtx + dL_dpy * dpy_dtx;
    const float dty = dL_dpx * 0.0f + dL_dpy * dpy_dty;
    const float dtz = dL_dpx * dpx_dtz + dL_dpy * dpy_dtz;
    const float3 dm = xform_vec_T(float3{dtx, dty, dtz}, vm);
    dL_dmeans = dL_dmeans + v3(dm.x, dm.y, dm.z);
  }

  // ---- computeColorFromSH backward (backward.cu:30-151) ----
  if (p.shs != nullptr && dsh != nullptr) {
    const int deg = p.D;
    const V3 pos = v3(mean.x, mean.y, mean.z);
    const V3 campos = v3(p.campos[0], p.campos[1], p.campos[2]);
    const V3 dir_orig = pos - campos;
    const V3 dir = dir_orig / sqrtf(dot3(dir_orig, dir_orig));
    const float* shg = p.shs + (size_t)idx * M * 3;
    auto sh = [shg](int k) { return v3(__ldg(shg + 3 * k), __ldg(shg + 3 * k + 1), __ldg(shg + 3 * k + 2)); };
    const uint32_t clamp_bits = __float_as_uint(p.color[idx].w);
    V3 dL_dRGB = v3(dL_dcolor[0], dL_dcolor[1], dL_dcolor[2]);
    dL_dRGB.x *= (clamp_bits & 1u) ? 0 : 1;
    dL_dRGB.y *= (clamp_bits & 2u) ? 0 : 1;
    dL_dRGB.z *= (clamp_bits & 4u) ? 0 : 1;
    V3 dRGBdx = v3(0, 0, 0), dRGBdy = v3(0, 0, 0), dRGBdz = v3(0, 0, 0);
    const float x = dir.x, y = dir.y, z = dir.z;
    auto put = [dsh](int k, V3 g) {
      dsh[3 * k] = g.x;
      dsh[3 * k + 1] = g.y;
      dsh[3 * k + 2] = g.z;
    };
    int written = 1;
    const float dRGBdsh0 = kShC0;
    put(0, dRGBdsh0 * dL_dRGB);
    if (deg > 0) {
      const float dRGBdsh1 = -kShC1 * y;
      const float dRGBdsh2 = kShC1 * z;
      const float dRGBdsh3 = -kShC1 * x;
      put(1, dRGBdsh1 * dL_dRGB);
      put(2, dRGBdsh2 * dL_dRGB);
      put(3, dRGBdsh3 * dL_dRGB);
      written = 4;
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
        written = 9;
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
          written = 16;
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
    for (int k = written; k < M; ++k) put(k, v3(0.f, 0.f, 0.f));
    const V3 dL_ddir = v3(dot3(dRGBdx, dL_dRGB), dot3(dRGBdy, dL_dRGB), dot3(dRGBdz, dL_dRGB));
    const float3 dn = dnormvdv3(float3{dir_orig.x, dir_orig.y, dir_orig.z}, float3{dL_ddir.x, dL_ddir.y, dL_ddir.z});
    dL_dmeans = dL_dmeans + v3(dn.x, dn.y, dn.z);
  } else if (dsh != nullptr) {
    for (int k = 0; k < 3 * M; ++k) dsh[k] = 0.f;
  }
  p.dL_dmeans3D[3 * idx] = dL_dmeans.x;
  p.dL_dmeans3D[3 * idx + 1] = dL_dmeans.y;
  p.dL_dmeans3D[3 * idx + 2] = dL_dmeans.z;

  // ---- computeCov3D backward (backward.cu:489-552) ----
  if (p.scales != nullptr && p.cov3D_precomp == nullptr) {
    const float q_r = p.rotations[4 * idx], q_x = p.rotations[4 * idx + 1];
    const float q_y = p.rotations[4 * idx + 2], q_z = p.rotations[4 * idx + 3];
    const float r = q_r, x = q_x, y = q_y, z = q_z;
    const Mat3c R = mat3_cols(1.f - 2.f * (y * y + z * z), 2.f * (x * y - r * z), 2.f * (x * z + r * y),
                              2.f * (x * y + r * z), 1.f - 2.f * (x * x + z * z), 2.f * (y * z - r * x),
                              2.f * (x * z - r * y), 2.f * (y * z + r * x), 1.f - 2.f * (x * x + y * y));
    Mat3c S = mat3_identity();
    const float mod = p.scale_modifier;
    const V3 s = mod * v3(p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]);
    S.m[0][0] = s.x;
    S.m[1][1] = s.y;
    S.m[2][2] = s.z;
    const Mat3c Mm = mat3_mul(S, R);
    const float* d = dcov;
    const Mat3c dL_dSigma = mat3_cols(d[0], 0.5f * d[1], 0.5f * d[2], 0.5f * d[1], d[3], 0.5f * d[4],
                                      0.5f * d[2], 0.5f * d[4], d[5]);
    Mat3c twoM;
    for (int cc = 0; cc < 3; ++cc)
      for (int rr = 0; rr < 3; ++rr) twoM.m[cc][rr] = Mm.m[cc][rr] * 2.0f;
    const Mat3c dL_dM = mat3_mul(twoM, dL_dSigma);
    const Mat3c Rt = mat3_transpose(R);
    Mat3c dL_dMt = mat3_transpose(dL_dM);
    const float sx = Rt.m[0][0] * dL_dMt.m[0][0] + Rt.m[0][1] * dL_dMt.m[0][1] + Rt.m[0][2] * dL_dMt.m[0][2];
    const float sy = Rt.m[1][0] * dL_dMt.m[1][0] + Rt.m[1][1] * dL_dMt.m[1][1] + Rt.m[1][2] * dL_dMt.m[1][2];
    const float sz = Rt.m[2][0] * dL_dMt.m[2][0] + Rt.m[2][1] * dL_dMt.m[2][1] + Rt.m[2][2] * dL_dMt.m[2][2];
    p.dL_dscales[3 * idx] = sx;
    p.dL_dscales[3 * idx + 1] = sy;
    p.dL_dscales[3 * idx + 2] = sz;
    for (int rr = 0; rr < 3; ++rr) {
      dL_dMt.m[0][rr] *= s.x;
      dL_dMt.m[1][rr] *= s.y;
      dL_dMt.m[2][rr] *= s.z;
    }
    const auto& G = dL_dMt.m;
    p.dL_drotations[4 * idx] = 2 * z * (G[0][1] - G[1][0]) + 2 * y * (G[2][0] - G[0][2]) + 2 * x * (G[1][2] - G[2][1]);
    p.dL_drotations[4 * idx + 1] = 2 * y * (G[1][0] + G[0][1]) + 2 * z * (G[2][0] + G[0][2]) +
                                   2 * r * (G[1][2] - G[2][1]) - 4 * x * (G[2][2] + G[1][1]);
    p.dL_drotations[4 * idx + 2] = 2 * x * (G[1][0] + G[0][1]) + 2 * r * (G[2][0] - G[0][2]) +
                                   2 * z * (G[1][2] + G[2][1]) - 4 * y * (G[2][2] + G[0][0]);
    p.dL_drotations[4 * idx + 3] = 2 * r * (G[0][1] - G[1][0]) + 2 * x * (G[2][0] + G[0][2]) +
                                   2 * y * (G[1][2] + G[2][1]) - 4 * z * (G[1][1] + G[0][0]);
  } else {
    for (int k = 0; k < 3; ++k) p.dL_dscales[3 * idx + k] = 0.f;
    for (int k = 0; k < 4; ++k) p.dL_drotations[4 * idx + k] = 0.f;
  }
}

}  // namespace

void launch_preprocess_backward(const PreprocessBackwardParams& p, cudaStream_t s) {
  if (p.P <= 0) return;
  preprocess_backward_kernel<<<(p.P + 255) / 256, 256, 0, s>>>(p);
}

}  // namespace omnigs
