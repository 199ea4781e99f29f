// Backward of the lonlat preprocess, one thread per Gaussian, fused into one kernel.
//
// The reference runs two kernels and round-trips dL/dmeans3D and the Jacobian rows dpx_dt /
// dpy_dt through global memory (backward.cu:948-1016): computeCov2DLonLatCUDA (:297-485) then
// preprocessLonLatCUDA (:613-669) with the SH backward (:30-151) and the scale/rotation backward
// (:489-552).  Here one thread does all of it (in registers, its SH coefficients and their
// gradients in its shared-memory row: below), recomputes cov3D from scale and
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

// Blocks of 128 threads.  A warp whose 32 Gaussians all exist and carry 16 FP32 SH coefficients
// (16-byte aligned input and gradient) moves its 6 KB of SH through shared memory: cp.async copies
// issued at the start (512 contiguous bytes per instruction, no registers held while the
// covariance backward runs), the SH backward reading each coefficient from the Gaussian's row, and
// the gradients written back through the same rows and stored 512 contiguous bytes per instruction.
// Other warps read and write each Gaussian's coefficients on their own.  Measured on a B200 at 1M
// Gaussians: 0.161 -> 0.134 ms; copying the rows into registers before the SH backward instead
// measured 0.289 ms.
constexpr int kPbThreads = 128;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__global__ void __launch_bounds__(kPbThreads) preprocess_backward_kernel(PreprocessBackwardParams p) {
  __shared__ float4 s_stage[kPbThreads / 32][32 * kShStageStride];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int M = p.M;
  const int first = idx - lane;
  float4* stage = s_stage[warp];
  const bool staged = p.shs != nullptr && p.dL_dsh != nullptr && M == kMaxShCoeffs && first + 32 <= p.P &&
                      ((reinterpret_cast<uintptr_t>(p.shs) | reinterpret_cast<uintptr_t>(p.dL_dsh)) & 15) == 0;
  if (staged) {
    const float4* src = reinterpret_cast<const float4*>(p.shs) + (size_t)first * 12;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const int e = i * 32 + lane;
      const int gg = e / 12, part = e - gg * 12;
      cp_async16(stage + gg * kShStageStride + part, src + e);
    }
    cp_async_commit();
  }
  if (idx >= p.P) return;  // (never in a staged warp)
  float* dsh = (p.dL_dsh != nullptr && M > 0) ? p.dL_dsh + (size_t)idx * M * 3 : nullptr;
  const bool culled = !(p.radii[idx] > 0);

  V3 dL_dmeans = v3(0.f, 0.f, 0.f);
  float dcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float3 mean = {0.f, 0.f, 0.f};
  float dL_dcolor[3] = {0.f, 0.f, 0.f};
  if (culled) {
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
    if (!staged) {
      if (dsh)
        for (int k = 0; k < 3 * M; ++k) dsh[k] = 0.f;
      return;
    }
    // a culled lane of a staged warp takes part in the warp's SH steps below with zero gradients
  } else {
    // ---- consume the accumulator record of the backward blend ----
    const float4 g0 = p.grad_acc[3 * idx];
    const float4 g1 = p.grad_acc[3 * idx + 1];
    const float4 g2 = p.grad_acc[3 * idx + 2];
    // the blend sums w dx and w dy (turned into the mean terms by the opacity and the conic here)
    // and the conic terms (by the opacity), all without their constant factors (render_bwd.cu);
    // the conic and opacity are read before the record is cleared (the compiler cannot move loads of possibly aliasing memory past those
    // stores)
    const float4 sa = __ldg(&p.splat[2 * idx]);  // {x, y, conic a, conic b}
    const float4 sb = __ldg(&p.splat[2 * idx + 1]);  // {conic c, opacity, ...}
    const float conic_c = sb.x, opacity = sb.y;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    p.grad_acc[3 * idx] = z4;
    p.grad_acc[3 * idx + 1] = z4;
    p.grad_acc[3 * idx + 2] = z4;
    const float mx = opacity * fmaf(sa.z, g0.x, sa.w * g0.y), my = opacity * fmaf(sa.w, g0.x, conic_c * g0.y);
    const float dmean2D_x = -0.5f * (float)p.W * mx, dmean2D_y = -0.5f * (float)p.H * my;
    const float ho = -0.5f * opacity;
    const float3 dL_dconic = {ho * g0.z, ho * g0.w, ho * g1.x};
    dL_dcolor[0] = g1.z;
    dL_dcolor[1] = g1.w;
    dL_dcolor[2] = g2.x;
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
    mean = {p.means3D[3 * idx], p.means3D[3 * idx + 1], p.means3D[3 * idx + 2]};
    float cov3D[6];
    if (p.cov3D_precomp != nullptr) {
      for (int k = 0; k < 6; ++k) cov3D[k] = p.cov3D_precomp[6 * idx + k];
    } else {
      const float3 s = {p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]};
      const float4 q = {p.rotations[4 * idx], p.rotations[4 * idx + 1], p.rotations[4 * idx + 2],
                        p.rotations[4 * idx + 3]};
      cov3d_from_scale_rot(s, p.scale_modifier, q, cov3D);
    }
    LonlatJacobian jac;
    dL_dmeans = cov2d_lonlat_backward<float>(mean, cov3D, vm, p.W, p.H, dL_dconic, dcov, jac);
    for (int k = 0; k < 6; ++k) p.dL_dcov3D[6 * idx + k] = dcov[k];

    // ---- preprocessLonLatCUDA: screen-space mean path (backward.cu:640-660) ----
    dL_dmeans = dL_dmeans + mean2d_backward(jac, dmean2D_x, dmean2D_y, p.W, p.H, vm);
  }

  // ---- computeColorFromSH backward (backward.cu:30-151) ----
  const int deg = p.D;
  auto sh_grad = [&](const float* shv, float dshv[3 * kMaxShCoeffs]) {
    auto sh = [&](int k) { return v3(shv[3 * k], shv[3 * k + 1], shv[3 * k + 2]); };
    auto put = [&](int k, V3 g) {
      dshv[3 * k] = g.x;
      dshv[3 * k + 1] = g.y;
      dshv[3 * k + 2] = g.z;
    };
    const uint32_t clamp_bits = __float_as_uint(p.color[idx].w);
    dL_dmeans = dL_dmeans + sh_backward(deg, v3(mean.x, mean.y, mean.z),
                                        v3(p.campos[0], p.campos[1], p.campos[2]), sh, clamp_bits,
                                        v3(dL_dcolor[0], dL_dcolor[1], dL_dcolor[2]), put);
  };
  if (staged) {
    cp_async_wait_all();
    __syncwarp();  // every lane's copies have landed
    float dshv[3 * kMaxShCoeffs];
    const int ncoef = culled ? 0 : (deg + 1) * (deg + 1);
    if (!culled) sh_grad(reinterpret_cast<const float*>(stage + lane * kShStageStride), dshv);
    __syncwarp();  // the warp's reads of the rows are done before they are overwritten
    float4* row = stage + lane * kShStageStride;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      float4 f;
      f.x = (4 * i < 3 * ncoef) ? dshv[4 * i] : 0.f;
      f.y = (4 * i + 1 < 3 * ncoef) ? dshv[4 * i + 1] : 0.f;
      f.z = (4 * i + 2 < 3 * ncoef) ? dshv[4 * i + 2] : 0.f;
      f.w = (4 * i + 3 < 3 * ncoef) ? dshv[4 * i + 3] : 0.f;
      row[i] = f;
    }
    __syncwarp();
    float4* dst = reinterpret_cast<float4*>(p.dL_dsh) + (size_t)first * 12;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const int e = i * 32 + lane;
      const int gg = e / 12, part = e - gg * 12;
      dst[e] = stage[gg * kShStageStride + part];
    }
    if (culled) return;
  } else if (p.shs != nullptr && dsh != nullptr) {
    float shv[3 * kMaxShCoeffs], dshv[3 * kMaxShCoeffs];
    load_sh<false>(p.shs, idx, M, shv);
    sh_grad(shv, dshv);
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
  preprocess_backward_kernel<<<(p.P + kPbThreads - 1) / kPbThreads, kPbThreads, 0, s>>>(p);
}

}  // namespace omnigs
