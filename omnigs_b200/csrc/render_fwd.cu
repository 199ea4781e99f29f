// Forward front-to-back alpha blend of one 16x16 tile per block (forward.cu:346-467).
//
// Every pixel evaluates exactly the reference's per-pair arithmetic and control flow (power,
// alpha = min(0.99, o exp(power)), the 1/255 skip, the T < 1e-4 stop), so the image, final
// transmittance and last-contributor index are identical for the same sorted instance list.
// What changes is the work around it:
//  * a thread owns two pixels of one column (rows 4 apart), a warp an 8 x 8 patch; the per-splat
//    shared-memory reads, loop control and votes are paid once per thread, not once per pixel,
//    and the two pixels' arithmetic runs in packed f32x2 instructions (each lane rounded exactly
//    as the scalar operation, so results are unchanged);
//  * for each staged batch a warp ballots which splats can reach alpha >= 1/255 somewhere in its
//    patch (the exact minimum of the splat's quadratic form over the patch against a threshold
//    computed in the preprocess) and iterates only over those, so pairs that the reference rejects
//    pixel by pixel are skipped a warp at a time;
//  * a warp stops after the group of 32 candidate splats in which all of its pixels saturated
//    (one warp vote per group; saturated pixels skip the per-splat work at once), and the block
//    stops when every warp has (block vote), as in the reference;
//  * splat geometry and colour are staged together (three float4 per instance) so the inner loop
//    reads only shared memory.
#include "blend_common.cuh"

namespace omnigs {
namespace {

template <int kBatch, bool kWrap>
__device__ __forceinline__ void blend_forward_tile(const TileJob& job, const BlendSource& src) {
  __shared__ float4 s_a[kBatch];  // x, y, conic a, conic b
  __shared__ float4 s_b[kBatch];  // conic c, opacity, cull threshold, conic determinant
  __shared__ float4 s_c[kBatch];  // r, g, b, clamp bits
  const BlendPatch patch = BlendPatch::make(job.tile_x, job.tile_y, job.wrap_w);
  float2 T, C0, C1, C2;
  uint32_t lc0, lc1;
  forward_pass<kBatch, kWrap, true>(job, src, patch, s_a, s_b, s_c, T, lc0, lc1, C0, C1, C2);

  const int64_t HW = (int64_t)job.H * job.W;
  const float Ts[2] = {T.x, T.y}, Cs[3][2] = {{C0.x, C0.y}, {C1.x, C1.y}, {C2.x, C2.y}};
  const uint32_t lcs[2] = {lc0, lc1};
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    if (!patch.inside(i, job.W, job.H)) continue;
    const int64_t pix = patch.pixel(i, job.W);
    if (job.final_T != nullptr) {  // stored unless the backward recomputes it
      job.final_T[pix] = Ts[i];
      job.n_contrib[pix] = lcs[i];
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) job.out_color[ch * HW + pix] = __fmaf_rn(Ts[i], job.bg[ch], Cs[ch][i]);
  }
}

// One view: block (x, y) blends tile (x, y).
template <int kBatch>
// Twelve resident blocks per SM (at most 40 registers) measured fastest for the single-view kernel
// on a B200 (0.511 -> 0.491 ms per 1M-Gaussian 2048x1024 view); the batched kernel measured
// marginally slower under the same bound and keeps the compiler's choice.
__global__ void __launch_bounds__(kBlendThreads, 12) render_forward_kernel(RenderParams p) {
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
  job.wrap_w = 0.f;
  blend_forward_tile<kBatch, false>(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P, p.capacity});
}

// All views of a batch in one launch: block b blends global tile b.
template <int kBatch, bool kWrap>
__global__ void __launch_bounds__(kBlendThreads) batch_render_forward_kernel(const __grid_constant__ BatchRenderParams p) {
  const TileJob job = batch_tile_job(p, blockIdx.x);
  blend_forward_tile<kBatch, kWrap>(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P * (uint32_t)p.V, p.capacity});
}

template <bool kWrap>
void launch_batch_blend(const BatchRenderParams& p, cudaStream_t s) {
  switch (blend_batch_size(false)) {
    case 128: batch_render_forward_kernel<128, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
    case 512: batch_render_forward_kernel<512, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
    default: batch_render_forward_kernel<256, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
  }
}

}  // namespace

void launch_render_forward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  const dim3 grid(p.gx, p.gy);
  switch (blend_batch_size(false)) {
    case 128: render_forward_kernel<128><<<grid, kBlendThreads, 0, s>>>(p); break;
    case 512: render_forward_kernel<512><<<grid, kBlendThreads, 0, s>>>(p); break;
    default: render_forward_kernel<256><<<grid, kBlendThreads, 0, s>>>(p); break;
  }
}

void launch_batch_render_forward(const BatchRenderParams& p, cudaStream_t s) {
  if (p.total_tiles == 0) return;
  if (p.seam_wrap)
    launch_batch_blend<true>(p, s);
  else
    launch_batch_blend<false>(p, s);
}

}  // namespace omnigs
