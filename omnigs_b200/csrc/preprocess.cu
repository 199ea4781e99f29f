// Forward preprocess of lonlat splats of one view, one thread per Gaussian.
//
// Evaluates the reference's FP32 sequence (forward.cu:592-703, preprocess_common.cuh): near cull at
// r^2 <= 0.04, equirect projection, 3D and 2D covariance, conic, radius, clamped tile rect and SH
// colour.  Outputs per Gaussian: radius, the 32-byte splat record and colour record read by the blend
// kernels, the radial depth (+inf for culled Gaussians: it is the depth-sort key of the binning)
// and tiles_touched; the instance total is summed on the device (block reduction + one atomic
// per block), so nothing is copied to the host (the reference copies num_rendered back between
// its scan and its duplication, rasterizer_impl.cu:622-628).
//
// Besides the reference's outputs, each visible splat gets the threshold of its quadratic form
// beyond which its alpha is provably below 1/255 and its conic's determinant; the blend kernels use
// them to skip a splat for a whole warp without changing any per-pixel decision.
#include "kernels.h"
#include "preprocess_common.cuh"
#include "sh_io.cuh"

namespace omnigs {
namespace {

// 128 threads: the per-warp SH stage (6.5 KB) of four warps.  Six resident blocks per SM (at most
// 85 registers) measured fastest on a B200 (0.102 -> 0.078 ms at 1M Gaussians with the staging).
constexpr int kPrepBlock = 128;

__global__ void __launch_bounds__(kPrepBlock, 6) preprocess_kernel(PreprocessParams p) {
  __shared__ uint32_t s_warp[kPrepBlock / 32];
  __shared__ float4 s_sh[kPrepBlock / 32][32 * kShStageStride];
  const int idx = blockIdx.x * kPrepBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool staged = warp_stage_sh(p.shs, idx - lane, p.P, p.M, s_sh[warp], lane);

  uint32_t touched = 0;
  if (idx < p.P) {
    const float3 p_orig = {p.means3D[3 * idx], p.means3D[3 * idx + 1], p.means3D[3 * idx + 2]};
    auto cov3d = [&](float out[6]) {
      if (p.cov3D_precomp != nullptr) {
#pragma unroll
        for (int k = 0; k < 6; ++k) out[k] = p.cov3D_precomp[6 * idx + k];
      } else {
        const float3 s = {p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]};
        const float4 q = {p.rotations[4 * idx], p.rotations[4 * idx + 1], p.rotations[4 * idx + 2],
                          p.rotations[4 * idx + 3]};
        cov3d_from_scale_rot(s, p.scale_modifier, q, out);
      }
    };
    float shv[3 * kMaxShCoeffs];
    if (staged)
      read_staged_sh(s_sh[warp], lane, shv);
    else if (p.shs != nullptr)
      load_sh<false>(p.shs, idx, p.M, shv);
    auto sh = [&](int k) { return v3(shv[3 * k], shv[3 * k + 1], shv[3 * k + 2]); };
    const SplatResult r = preprocess_splat</*kFp64Poles=*/false>(
        p_orig, p.viewmatrix, p.W, p.H, p.gx, p.gy, p.D, p.campos, p.opacities[idx],
        p.colors_precomp != nullptr ? p.colors_precomp + 3 * idx : nullptr, /*seam_wrap=*/false, cov3d, sh);
    p.radii[idx] = r.radius;
    if (r.radius > 0) {
      p.splat[2 * idx] = r.s0;
      p.splat[2 * idx + 1] = r.s1;
      p.color[idx] = r.col;
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      p.grad_acc[3 * idx] = z4;
      p.grad_acc[3 * idx + 1] = z4;
      p.grad_acc[3 * idx + 2] = z4;
    }
    p.depth[idx] = r.depth_key;
    p.tiles_touched[idx] = r.touched;
    touched = r.touched;
  }

  // ---- instance total: block reduction, one atomic per block ----
  uint32_t v = touched;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  if (lane == 0) s_warp[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long total = 0;
#pragma unroll
    for (int w = 0; w < kPrepBlock / 32; ++w) total += s_warp[w];
    if (total) atomicAdd(&p.hdr->num_rendered64, total);
  }
}

}  // namespace

void launch_preprocess(const PreprocessParams& p, cudaStream_t s) {
  if (p.P <= 0) return;
  const int blocks = (p.P + kPrepBlock - 1) / kPrepBlock;
  preprocess_kernel<<<blocks, kPrepBlock, 0, s>>>(p);
}

}  // namespace omnigs
