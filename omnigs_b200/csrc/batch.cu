// Batched multi-view preprocess, forward and backward: V equirect views of one shared Gaussian set.
//
// One thread per Gaussian reads the Gaussian's parameters once (mean, scale, rotation, opacity and
// its SH coefficients, FP32 or BF16, with 16-byte vector loads) and loops over the views:
//  * forward: for each view it evaluates the same per-(view, Gaussian) body as the single-view
//    preprocess (preprocess_common.cuh) and writes the view's splat, colour, depth and radius
//    records (view-major, record v * P + g) and zeroes the record's gradient accumulator; per-view
//    and total instance counts are summed on the device (no host synchronisation);
//  * backward: for each view where the Gaussian is visible it consumes the accumulator record the
//    backward blend wrote and runs the single-view backward pieces (preprocess_bwd_common.cuh),
//    summing dL/dmean3D, dL/dSH, dL/dopacity and dL/dcov3D over the views in registers; dL/dscale
//    and dL/drot follow once from the summed dL/dcov3D (the covariance backward is linear), and the
//    trainer's densification statistics (per-view |dL/dmean2D| sums, visible-view counts, maximum
//    radius) are accumulated in the same pass.
// So the parameters are read once per batch instead of once per view, and the parameter gradients
// are written once, already summed.
//
// Precision mode (template flags): SH read as BF16 (colour and gradients still accumulate in FP32)
// and FP64 for the 2D covariance, its inverse and its backward beyond 85 degrees of latitude.
#include "kernels.h"
#include "preprocess_bwd_common.cuh"
#include "preprocess_common.cuh"
#include "sh_io.cuh"

namespace omnigs {
namespace {

constexpr int kBatchBlock = 128;

// The Gaussian's 3D covariance: precomputed, or from scale and rotation (forward.cu:194-228).
__device__ __forceinline__ void gaussian_cov3d(const BatchParams& p, int g, float out[6]) {
  if (p.cov3D_precomp != nullptr) {
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = p.cov3D_precomp[6 * g + k];
  } else {
    const float3 s = {p.scales[3 * g], p.scales[3 * g + 1], p.scales[3 * g + 2]};
    const float4 q = {p.rotations[4 * g], p.rotations[4 * g + 1], p.rotations[4 * g + 2], p.rotations[4 * g + 3]};
    cov3d_from_scale_rot(s, p.scale_modifier, q, out);
  }
}

template <bool kFp64Poles, bool kShBf16>
__global__ void __launch_bounds__(kBatchBlock) batch_preprocess_kernel(const __grid_constant__ BatchParams p) {
  __shared__ uint32_t s_count[kMaxBatchViews][kBatchBlock / 32];
  const int g = blockIdx.x * kBatchBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool active = g < p.P;

  float3 p_orig = {0.f, 0.f, 0.f};
  float cov3D[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float shv[3 * kMaxShCoeffs];
  float opacity = 0.f;
  if (active) {
    p_orig = make_float3(p.means3D[3 * g], p.means3D[3 * g + 1], p.means3D[3 * g + 2]);
    gaussian_cov3d(p, g, cov3D);
    opacity = p.opacities[g];
    if (p.shs != nullptr) load_sh<kShBf16>(p.shs, g, p.M, shv);
  }
  auto cov3d = [&](float out[6]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = cov3D[k];
  };
  auto sh = [&](int k) { return v3(shv[3 * k], shv[3 * k + 1], shv[3 * k + 2]); };
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);

#pragma unroll 1
  for (int v = 0; v < p.V; ++v) {
    uint32_t touched = 0;
    if (active) {
      const BatchView& bv = p.views[v];
      const SplatResult r = preprocess_splat<kFp64Poles>(
          p_orig, p.viewmatrices + 16 * v, bv.W, bv.H, bv.gx, bv.gy, p.D, p.campos + 3 * v, opacity,
          p.colors_precomp != nullptr ? p.colors_precomp + 3 * g : nullptr, p.seam_wrap != 0, cov3d, sh);
      const size_t rec = (size_t)v * p.P + g;
      p.radii[rec] = r.radius;
      p.depth[rec] = r.depth_key;
      if (r.radius > 0) {
        p.splat[2 * rec] = r.s0;
        p.splat[2 * rec + 1] = r.s1;
        p.color[rec] = r.col;
        p.grad_acc[3 * rec] = z4;
        p.grad_acc[3 * rec + 1] = z4;
        p.grad_acc[3 * rec + 2] = z4;
      }
      touched = r.touched;
    }
    const uint32_t wsum = __reduce_add_sync(kFullMask, touched);
    if (lane == 0) s_count[v][warp] = wsum;
  }
  __syncthreads();
  // per-view and total instance counts: one atomic per view and block
  uint32_t mine = 0;
  if (threadIdx.x < p.V) {
#pragma unroll
    for (int w = 0; w < kBatchBlock / 32; ++w) mine += s_count[threadIdx.x][w];
    if (mine) atomicAdd(&p.view_rendered[threadIdx.x], (unsigned long long)mine);
  }
  if (warp == 0) {
    const uint32_t total = __reduce_add_sync(kFullMask, mine);
    if (lane == 0 && total) atomicAdd(&p.hdr->num_rendered64, (unsigned long long)total);
  }
}

// Three resident blocks per SM (at most 170 registers) for the FP32 arithmetic: 1.21 -> 0.92 ms per
// 16-view step over 1M Gaussians on a B200, against the 190 registers (two blocks) the compiler
// takes unbounded; the FP64-pole instantiations would spill heavily under that bound and keep theirs.
template <bool kFp64Poles>
constexpr int batch_bwd_min_blocks() { return kFp64Poles ? 1 : 3; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

// A warp whose 32 Gaussians all exist and carry 16 SH coefficients (16-byte aligned) copies its
// coefficients into shared memory with cp.async (512 contiguous bytes per instruction) and the SH
// backward of every view reads them from the Gaussian's row, instead of 48 registers per thread
// (0.979 -> 0.942 ms per 16-view step over 1M Gaussians on a B200).
template <bool kFp64Poles, bool kShBf16>
__global__ void __launch_bounds__(kBatchBlock, batch_bwd_min_blocks<kFp64Poles>())
    batch_preprocess_backward_kernel(const __grid_constant__ BatchParams p, const BatchGrads out) {
  constexpr int kRowU4 = kShBf16 ? 6 : 12;  // 16-byte pieces of a Gaussian's coefficients
  constexpr int kStrideU4 = kRowU4 + 1;     // odd: a quarter-warp's 16-byte row reads hit distinct banks
  __shared__ uint4 s_stage[kBatchBlock / 32][32 * kStrideU4];
  const int g = blockIdx.x * kBatchBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int first = g - lane;
  const bool with_sh = p.shs != nullptr;
  const bool staged = with_sh && p.M == kMaxShCoeffs && first + 32 <= p.P &&
                      (reinterpret_cast<uintptr_t>(p.shs) & 15) == 0;
  uint4* stage = s_stage[warp];
  if (staged) {
    const uint4* src = reinterpret_cast<const uint4*>(p.shs) + (size_t)first * kRowU4;
#pragma unroll
    for (int i = 0; i < kRowU4; ++i) {
      const int e = i * 32 + lane;
      const int gg = e / kRowU4, part = e - gg * kRowU4;
      cp_async16(stage + gg * kStrideU4 + part, src + e);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  if (g >= p.P) return;  // (never in a staged warp)
  const float3 mean = {p.means3D[3 * g], p.means3D[3 * g + 1], p.means3D[3 * g + 2]};
  float cov3D[6];
  gaussian_cov3d(p, g, cov3D);
  if (staged) {
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();  // every lane's copies have landed
  }
  // the rest of the kernel, given the accessor of the Gaussian's coefficients
  auto finish = [&](auto sh) {
  float dsh[3 * kMaxShCoeffs];
#pragma unroll
  for (int k = 0; k < 3 * kMaxShCoeffs; ++k) dsh[k] = 0.f;
  auto put = [&](int k, V3 d) {
    dsh[3 * k] += d.x;
    dsh[3 * k + 1] += d.y;
    dsh[3 * k + 2] += d.z;
  };

  V3 dmean = v3(0.f, 0.f, 0.f), dcolor = v3(0.f, 0.f, 0.f);
  float dcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float dopacity = 0.f, stat_norm = 0.f, stat_views = 0.f;
  int max_radius = 0;
#pragma unroll 1
  for (int v = 0; v < p.V; ++v) {
    const size_t rec = (size_t)v * p.P + g;
    const int radius = p.radii[rec];
    if (!(radius > 0)) continue;
    const float4 g0 = p.grad_acc[3 * rec];
    const float4 g1 = p.grad_acc[3 * rec + 1];
    const float4 g2 = p.grad_acc[3 * rec + 2];
    const float* vm = p.viewmatrices + 16 * v;
    const int W = p.views[v].W, H = p.views[v].H;
    // the blend sums w dx and w dy (turned into the mean terms by the opacity and the conic here)
    // and the conic terms (by the opacity), all without their constant factors (render_bwd.cu)
    const float4 sa = p.splat[2 * rec];  // {x, y, conic a, conic b}
    const float4 sb = p.splat[2 * rec + 1];  // {conic c, opacity, ...}
    const float conic_c = sb.x, opacity = sb.y;
    const float mx = opacity * fmaf(sa.z, g0.x, sa.w * g0.y), my = opacity * fmaf(sa.w, g0.x, conic_c * g0.y);
    const float ho = -0.5f * opacity;
    const float3 dconic = {ho * g0.z, ho * g0.w, ho * g1.x};
    const float dm2x = -0.5f * (float)W * mx, dm2y = -0.5f * (float)H * my;
    float dcov_v[6];
    LonlatJacobian jac;
    V3 dm;
    bool pole = false;
    if (kFp64Poles) {
      const float3 t = xform_point(mean, vm);
      pole = fabsf(t.y) > kPoleSinLat * sqrtf(t.x * t.x + t.y * t.y + t.z * t.z);
    }
    if (pole)
      dm = cov2d_lonlat_backward<double>(mean, cov3D, vm, W, H, dconic, dcov_v, jac);
    else
      dm = cov2d_lonlat_backward<float>(mean, cov3D, vm, W, H, dconic, dcov_v, jac);
#pragma unroll
    for (int k = 0; k < 6; ++k) dcov[k] += dcov_v[k];
    dm = dm + mean2d_backward(jac, dm2x, dm2y, W, H, vm);
    const V3 dcol = v3(g1.z, g1.w, g2.x);
    if (with_sh) {
      const float* cp = p.campos + 3 * v;
      dm = dm + sh_backward(p.D, v3(mean.x, mean.y, mean.z), v3(cp[0], cp[1], cp[2]), sh,
                            __float_as_uint(p.color[rec].w), dcol, put);
    }
    dmean = dmean + dm;
    dcolor = dcolor + dcol;
    dopacity += g1.y;
    stat_norm += sqrtf(dm2x * dm2x + dm2y * dm2y);
    stat_views += 1.f;
    max_radius = max(max_radius, radius);
  }

  out.dL_dmeans3D[3 * g] = dmean.x;
  out.dL_dmeans3D[3 * g + 1] = dmean.y;
  out.dL_dmeans3D[3 * g + 2] = dmean.z;
  out.dL_dopacity[g] = dopacity;
  if (out.dL_dsh != nullptr && p.M > 0)
    store_sh_grad(out.dL_dsh + (size_t)g * p.M * 3, p.M, with_sh ? (p.D + 1) * (p.D + 1) : 0, dsh);
  if (p.scales != nullptr && p.cov3D_precomp == nullptr) {
    const float3 s = {p.scales[3 * g], p.scales[3 * g + 1], p.scales[3 * g + 2]};
    const float4 q = {p.rotations[4 * g], p.rotations[4 * g + 1], p.rotations[4 * g + 2], p.rotations[4 * g + 3]};
    float dscale[3], drot[4];
    cov3d_backward(s, p.scale_modifier, q, dcov, dscale, drot);
    for (int k = 0; k < 3; ++k) out.dL_dscales[3 * g + k] = dscale[k];
    for (int k = 0; k < 4; ++k) out.dL_drotations[4 * g + k] = drot[k];
  } else {
    for (int k = 0; k < 3; ++k) out.dL_dscales[3 * g + k] = 0.f;
    for (int k = 0; k < 4; ++k) out.dL_drotations[4 * g + k] = 0.f;
  }
  if (out.dL_dcov3D != nullptr)
    for (int k = 0; k < 6; ++k) out.dL_dcov3D[6 * g + k] = dcov[k];
  if (out.dL_dcolors != nullptr) {
    out.dL_dcolors[3 * g] = dcolor.x;
    out.dL_dcolors[3 * g + 1] = dcolor.y;
    out.dL_dcolors[3 * g + 2] = dcolor.z;
  }
  if (stat_views > 0.f) {
    if (out.grad_accum != nullptr) out.grad_accum[g] += stat_norm;
    if (out.denom != nullptr) out.denom[g] += stat_views;
    if (out.max_radii != nullptr) out.max_radii[g] = fmaxf(out.max_radii[g], (float)max_radius);
  }
  };
  if (staged) {
    const uint4* my_row = stage + lane * kStrideU4;
    auto coef = [&](int c) -> float {
      if (kShBf16) return __uint_as_float((uint32_t)reinterpret_cast<const uint16_t*>(my_row)[c] << 16);
      return reinterpret_cast<const float*>(my_row)[c];
    };
    finish([&](int k) { return v3(coef(3 * k), coef(3 * k + 1), coef(3 * k + 2)); });
  } else {
    float shv[3 * kMaxShCoeffs];
    if (with_sh) load_sh<kShBf16>(p.shs, g, p.M, shv);
    finish([&](int k) { return v3(shv[3 * k], shv[3 * k + 1], shv[3 * k + 2]); });
  }
}

template <bool kFp64Poles, bool kShBf16>
void launch_preprocess_pair(const BatchParams& p, const BatchGrads* g, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.P + kBatchBlock - 1) / kBatchBlock);
  if (g == nullptr)
    batch_preprocess_kernel<kFp64Poles, kShBf16><<<blocks, kBatchBlock, 0, s>>>(p);
  else
    batch_preprocess_backward_kernel<kFp64Poles, kShBf16><<<blocks, kBatchBlock, 0, s>>>(p, *g);
}

void dispatch(const BatchParams& p, const BatchGrads* g, int fp64_poles, cudaStream_t s) {
  if (p.P <= 0 || p.V <= 0) return;
  const bool bf16 = p.sh_bf16 != 0 && p.shs != nullptr;
  if (fp64_poles) {
    if (bf16)
      launch_preprocess_pair<true, true>(p, g, s);
    else
      launch_preprocess_pair<true, false>(p, g, s);
  } else {
    if (bf16)
      launch_preprocess_pair<false, true>(p, g, s);
    else
      launch_preprocess_pair<false, false>(p, g, s);
  }
}

}  // namespace

void launch_batch_preprocess(const BatchParams& p, int fp64_poles, cudaStream_t s) {
  dispatch(p, nullptr, fp64_poles, s);
}

void launch_batch_preprocess_backward(const BatchParams& p, const BatchGrads& g, int fp64_poles, cudaStream_t s) {
  dispatch(p, &g, fp64_poles, s);
}

}  // namespace omnigs
