// Forward front-to-back alpha blend of one 16x16 tile per block (forward.cu:346-467).
//
// Every pixel evaluates exactly the reference's per-pair arithmetic and control flow (power,
// alpha = min(0.99, o exp(power)), the 1/255 skip, the T < 1e-4 stop), so the image, final
// transmittance and last-contributor index are identical for the same sorted instance list.
// What changes is the work around it:
//  * a thread owns kBlendPx pixels of one column (rows 4 apart), a warp an 8 x (4 kBlendPx) patch;
//    the per-splat shared-memory reads, loop control and votes are paid once per thread, not
//    once per pixel, and the thread's pixels give the scheduler independent work;
//  * for each staged batch a warp ballots which splats' alpha-support boxes (computed in the
//    preprocess) touch its patch and iterates only over those, so pairs that the reference rejects
//    pixel by pixel are skipped a warp at a time;
//  * a warp stops as soon as all of its pixels are saturated (warp vote), and the block stops when
//    every warp has (block vote), as in the reference;
//  * splat geometry and colour are staged together (three float4 per instance) so the inner loop
//    reads only shared memory.
#include "blend_common.cuh"

namespace omnigs {
namespace {

__device__ __forceinline__ void blend_forward_tile(const TileJob& job, const BlendSource& src) {
  __shared__ float4 s_a[kBatch];  // x, y, conic a, conic b
  __shared__ float4 s_b[kBatch];  // conic c, opacity, cull half-width, cull half-height
  __shared__ float4 s_c[kBatch];  // r, g, b, clamp bits
  const BlendPatch patch = BlendPatch::make(job.tile_x, job.tile_y);
  const int lane = threadIdx.x & 31;
  const uint2 range = job.range;
  const int n = (int)(range.y - range.x);

  bool done[kBlendPx];
  float T[kBlendPx], C0[kBlendPx], C1[kBlendPx], C2[kBlendPx];
  uint32_t last_contributor[kBlendPx];
#pragma unroll
  for (int i = 0; i < kBlendPx; ++i) {
    done[i] = !patch.inside(i, job.W, job.H);
    T[i] = 1.0f;
    C0[i] = C1[i] = C2[i] = 0.f;
    last_contributor[i] = 0;
  }
  auto all_done = [&] {
    bool d = true;
#pragma unroll
    for (int i = 0; i < kBlendPx; ++i) d = d && done[i];
    return d;
  };

  for (int base = 0; base < n; base += kBatch) {
    if (__syncthreads_and(all_done())) break;
    stage_batch(src, range.x, base, min(kBatch, n - base), /*reverse=*/false, s_a, s_b, s_c, nullptr);
    __syncthreads();
    const int cnt = min(kBatch, n - base);
    bool warp_done = __all_sync(kFullMask, all_done());
    for (int k = 0; k * 32 < cnt && !warp_done; ++k) {
      const int j = k * 32 + lane;
      bool hit = false;
      if (j < cnt) hit = patch.hit(s_a[j], s_b[j]);
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        const float4 a = s_a[jj];
        const float4 b = s_b[jj];
#pragma unroll
        for (int i = 0; i < kBlendPx; ++i) {
          if (done[i]) continue;
          const float2 d = {a.x - patch.pxf, a.y - patch.pyf(i)};
          const float power = splat_power(a, b, d);
          if (power > 0.0f) continue;
          const float alpha = fminf(0.99f, b.y * expf(power));
          if (alpha < 1.0f / 255.0f) continue;
          const float test_T = T[i] * (1 - alpha);
          if (test_T < 0.0001f) {
            done[i] = true;
            continue;
          }
          const float4 c = s_c[jj];
          // C += colour * alpha * T, rounded as the reference's compiled blend (fused add)
          C0[i] = __fmaf_rn(__fmul_rn(c.x, alpha), T[i], C0[i]);
          C1[i] = __fmaf_rn(__fmul_rn(c.y, alpha), T[i], C1[i]);
          C2[i] = __fmaf_rn(__fmul_rn(c.z, alpha), T[i], C2[i]);
          T[i] = test_T;
          last_contributor[i] = (uint32_t)(base + jj + 1);
        }
        if (__all_sync(kFullMask, all_done())) {
          warp_done = true;
          break;
        }
      }
    }
  }

  const int64_t HW = (int64_t)job.H * job.W;
#pragma unroll
  for (int i = 0; i < kBlendPx; ++i) {
    if (!patch.inside(i, job.W, job.H)) continue;
    const int64_t pix = patch.pixel(i, job.W);
    job.final_T[pix] = T[i];
    job.n_contrib[pix] = last_contributor[i];
    job.out_color[pix] = __fmaf_rn(T[i], job.bg[0], C0[i]);
    job.out_color[HW + pix] = __fmaf_rn(T[i], job.bg[1], C1[i]);
    job.out_color[2 * HW + pix] = __fmaf_rn(T[i], job.bg[2], C2[i]);
  }
}

// One view: block (x, y) blends tile (x, y).
__global__ void __launch_bounds__(kBlendThreads) render_forward_kernel(RenderParams p) {
  TileJob job;
  job.tile_x = blockIdx.x;
  job.tile_y = blockIdx.y;
  job.W = p.W;
  job.H = p.H;
  job.range = checked_range(p.ranges, blockIdx.y * p.gx + blockIdx.x, p.capacity);
  job.bg = p.bg;
  job.out_color = p.out_color;
  job.final_T = p.final_T;
  job.n_contrib = p.n_contrib;
  job.dL_dpix = nullptr;
  blend_forward_tile(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P, p.capacity});
}

// All views of a batch in one launch: block b blends global tile b.
__global__ void __launch_bounds__(kBlendThreads) batch_render_forward_kernel(const __grid_constant__ BatchRenderParams p) {
  const TileJob job = batch_tile_job(p, blockIdx.x);
  blend_forward_tile(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P * (uint32_t)p.V, p.capacity});
}

}  // namespace

void launch_render_forward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  render_forward_kernel<<<dim3(p.gx, p.gy), kBlendThreads, 0, s>>>(p);
}

void launch_batch_render_forward(const BatchRenderParams& p, cudaStream_t s) {
  if (p.total_tiles == 0) return;
  batch_render_forward_kernel<<<p.total_tiles, kBlendThreads, 0, s>>>(p);
}

}  // namespace omnigs
