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
#include "preprocess_bwd_common.cuh"
#include "sh_io.cuh"

namespace omnigs {
namespace {

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
  // the blend sums q dx and q dy (turned into the mean terms by the conic here) and the conic
  // terms, all without their constant factors (render_bwd.cu); the conic is read before the record
  // is cleared (the compiler cannot move loads of possibly aliasing memory past those stores)
  const float4 sa = __ldg(&p.splat[2 * idx]);  // {x, y, conic a, conic b}
  const float conic_c = __ldg(&p.splat[2 * idx + 1].x);
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  p.grad_acc[3 * idx] = z4;
  p.grad_acc[3 * idx + 1] = z4;
  p.grad_acc[3 * idx + 2] = z4;
  const float mx = fmaf(sa.z, g0.x, sa.w * g0.y), my = fmaf(sa.w, g0.x, conic_c * g0.y);
  const float dmean2D_x = -0.5f * (float)p.W * mx, dmean2D_y = -0.5f * (float)p.H * my;
  const float3 dL_dconic = {-0.5f * g0.z, -0.5f * g0.w, -0.5f * g1.x};
  const float dL_dcolor[3] = {g1.z, g1.w, g2.x};
  p.dL_dmeans2D[3 * idx] = dmean2D_x;
  p.dL_dmeans2D[3 * idx + 1] = dmean2D_y;
  p.dL_dmeans2D[3 * idx + 2] = 0.f;
  if (p.dL_dconic) {
    p.dL_dconic[4 * idx] = dL_dconic.x;
    p.dL_dconic[4 * idx + 1] = dL_dconic.y;
    p.dL_dconic[4 * idx + 2] = 0.f;
    p.dL_dconic[4 * idx + 3] = dL_dconic.z;
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
  float dcov[6];
  LonlatJacobian jac;
  V3 dL_dmeans = cov2d_lonlat_backward<float>(mean, cov3D, vm, p.W, p.H, dL_dconic, dcov, jac);
  for (int k = 0; k < 6; ++k) p.dL_dcov3D[6 * idx + k] = dcov[k];

  // ---- preprocessLonLatCUDA: screen-space mean path (backward.cu:640-660) ----
  dL_dmeans = dL_dmeans + mean2d_backward(jac, dmean2D_x, dmean2D_y, p.W, p.H, vm);

  // ---- computeColorFromSH backward (backward.cu:30-151) ----
  if (p.shs != nullptr && dsh != nullptr) {
    float shv[3 * kMaxShCoeffs], dshv[3 * kMaxShCoeffs];
    load_sh<false>(p.shs, idx, M, shv);
    auto sh = [&](int k) { return v3(shv[3 * k], shv[3 * k + 1], shv[3 * k + 2]); };
    auto put = [&](int k, V3 g) {
      dshv[3 * k] = g.x;
      dshv[3 * k + 1] = g.y;
      dshv[3 * k + 2] = g.z;
    };
    const int deg = p.D;
    const uint32_t clamp_bits = __float_as_uint(p.color[idx].w);
    dL_dmeans = dL_dmeans + sh_backward(deg, v3(mean.x, mean.y, mean.z),
                                        v3(p.campos[0], p.campos[1], p.campos[2]), sh, clamp_bits,
                                        v3(dL_dcolor[0], dL_dcolor[1], dL_dcolor[2]), put);
    store_sh_grad(dsh, M, (deg + 1) * (deg + 1), dshv);
  } else if (dsh != nullptr) {
    for (int k = 0; k < 3 * M; ++k) dsh[k] = 0.f;
  }
  p.dL_dmeans3D[3 * idx] = dL_dmeans.x;
  p.dL_dmeans3D[3 * idx + 1] = dL_dmeans.y;
  p.dL_dmeans3D[3 * idx + 2] = dL_dmeans.z;

  // ---- computeCov3D backward (backward.cu:489-552) ----
  if (p.scales != nullptr && p.cov3D_precomp == nullptr) {
    const float3 s = {p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]};
    const float4 q = {p.rotations[4 * idx], p.rotations[4 * idx + 1], p.rotations[4 * idx + 2],
                      p.rotations[4 * idx + 3]};
    float dscale[3], drot[4];
    cov3d_backward(s, p.scale_modifier, q, dcov, dscale, drot);
    for (int k = 0; k < 3; ++k) p.dL_dscales[3 * idx + k] = dscale[k];
    for (int k = 0; k < 4; ++k) p.dL_drotations[4 * idx + k] = drot[k];
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
