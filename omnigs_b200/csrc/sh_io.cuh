// Vectorised SH coefficient I/O of one Gaussian: 16-byte loads of its coefficients into registers
// (FP32 or BF16 storage) and 16-byte stores of its coefficient gradients.  A thread owns one
// Gaussian's 48 floats (192 B, or 96 B in BF16), which per-float accesses would spread over 48
// load/store instructions.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace omnigs {

constexpr int kMaxShCoeffs = 16;

// Coefficients [0, 16) of Gaussian g (zeros beyond M) into out[48], RGB inner.
template <bool kShBf16>
__device__ __forceinline__ void load_sh(const void* shs, int g, int M, float out[3 * kMaxShCoeffs]) {
  const size_t off = (size_t)g * M * 3;
  if (kShBf16) {
    const __nv_bfloat16* base = static_cast<const __nv_bfloat16*>(shs) + off;
    if (M == kMaxShCoeffs && (reinterpret_cast<uintptr_t>(base) & 15) == 0) {
      const uint4* v = reinterpret_cast<const uint4*>(base);
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        const uint4 u = __ldg(v + i);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          out[8 * i + 2 * k] = __uint_as_float(w[k] << 16);
          out[8 * i + 2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3 * kMaxShCoeffs; ++i) out[i] = (i < 3 * M) ? __bfloat162float(base[i]) : 0.f;
    }
  } else {
    const float* base = static_cast<const float*>(shs) + off;
    if (M == kMaxShCoeffs && (reinterpret_cast<uintptr_t>(base) & 15) == 0) {
      const float4* v = reinterpret_cast<const float4*>(base);
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const float4 f = __ldg(v + i);
        out[4 * i] = f.x;
        out[4 * i + 1] = f.y;
        out[4 * i + 2] = f.z;
        out[4 * i + 3] = f.w;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3 * kMaxShCoeffs; ++i) out[i] = (i < 3 * M) ? __ldg(base + i) : 0.f;
    }
  }
}

// Warp-cooperative staging of FP32 SH (M == 16): the warp's 32 consecutive Gaussians own one
// contiguous 6 KB span, which the warp loads with 12 fully coalesced 16-byte loads per lane (each
// instruction reads 512 contiguous bytes) into `stage`, instead of each lane reading its own 192 B
// (every warp instruction then touches 32 separate cache lines).  `stage` holds kShStageStride
// float4 per Gaussian: the spare float4 puts the 16-byte reads of 8 lanes (one shared-memory
// phase) of their own records on distinct banks.  warp_stage_sh is warp-uniform; it returns false,
// loading nothing, unless the whole warp qualifies (full warp, M == 16, 16-byte aligned).
constexpr int kShStageStride = 13;

__device__ __forceinline__ bool warp_stage_sh(const float* shs, int first, int P, int M, float4* stage, int lane) {
  if (shs == nullptr || M != kMaxShCoeffs || first + 32 > P || (reinterpret_cast<uintptr_t>(shs) & 15) != 0)
    return false;
  const float4* src = reinterpret_cast<const float4*>(shs) + (size_t)first * 12;
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const int e = i * 32 + lane;
    const int gg = e / 12, part = e - gg * 12;
    stage[gg * kShStageStride + part] = __ldg(src + e);
  }
  __syncwarp();
  return true;
}

// This lane's 48 staged coefficients.
__device__ __forceinline__ void read_staged_sh(const float4* stage, int lane, float out[3 * kMaxShCoeffs]) {
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const float4 f = stage[lane * kShStageStride + i];
    out[4 * i] = f.x;
    out[4 * i + 1] = f.y;
    out[4 * i + 2] = f.z;
    out[4 * i + 3] = f.w;
  }
}

// Writes the gradient of Gaussian g's M coefficients at d (= dL_dsh + g M 3): v[3k + ch] for
// k < ncoef, zeros for the remaining coefficients.
__device__ __forceinline__ void store_sh_grad(float* d, int M, int ncoef, const float v[3 * kMaxShCoeffs]) {
  if (M == kMaxShCoeffs && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      float4 f;
      f.x = (4 * i < 3 * ncoef) ? v[4 * i] : 0.f;
      f.y = (4 * i + 1 < 3 * ncoef) ? v[4 * i + 1] : 0.f;
      f.z = (4 * i + 2 < 3 * ncoef) ? v[4 * i + 2] : 0.f;
      f.w = (4 * i + 3 < 3 * ncoef) ? v[4 * i + 3] : 0.f;
      reinterpret_cast<float4*>(d)[i] = f;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 3 * kMaxShCoeffs; ++i)
      if (i < 3 * M) d[i] = (i < 3 * ncoef) ? v[i] : 0.f;
    for (int i = 3 * kMaxShCoeffs; i < 3 * M; ++i) d[i] = 0.f;
  }
}

}  // namespace omnigs
