// Backward back-to-front blend of one 16x16 tile per block (backward.cu:672-843).
//
// Per pixel this replays the reference's recurrence: start from the stored final transmittance
// and last-contributor index, walk the tile's instances from the back, undo T /= (1 - alpha) and
// accumulate the colour-behind term.  (One correctly rounded reciprocal of 1 - alpha serves both
// of the reference's divisions by it.)  The per-(pixel, splat) gradients (2 screen-space mean, 3
// conic, 1 opacity, 3 colour) are not pushed with 9 global atomics per pixel as in the reference:
// a thread first sums them over its kBlendPx pixels, the warp that owns the 8 x (4 kBlendPx) patch
// reduces them with a reduce-scatter of 8 values (9 shuffles) plus a butterfly for the ninth, and
// 8 lanes add one accumulator record per splat; when a single lane contributes it adds its 9
// values directly.  Warps skip splats whose alpha-support box misses their patch or that lie
// behind all of their pixels' last contributors, and the block starts at the batch holding its
// largest last contributor instead of at the end of the range.
#include "blend_common.cuh"

namespace omnigs {
namespace {

// Sums v[0..8] over the warp and adds the totals to acc[0..8] (one accumulator record).
__device__ __forceinline__ void warp_reduce_add9(const float v[9], float* acc, int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float a[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float send = b4 ? v[i] : v[i + 4];
    const float keep = b4 ? v[i + 4] : v[i];
    a[i] = keep + __shfl_xor_sync(kFullMask, send, 16);
  }
  float b[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float send = b3 ? a[i] : a[i + 2];
    const float keep = b3 ? a[i + 2] : a[i];
    b[i] = keep + __shfl_xor_sync(kFullMask, send, 8);
  }
  float c;
  {
    const float send = b2 ? b[0] : b[1];
    const float keep = b2 ? b[1] : b[0];
    c = keep + __shfl_xor_sync(kFullMask, send, 4);
  }
  c += __shfl_xor_sync(kFullMask, c, 2);
  c += __shfl_xor_sync(kFullMask, c, 1);
  float e = v[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(kFullMask, e, o);
  // lane 4k now holds the total of value k
  if ((lane & 3) == 0) atomicAdd(acc + (lane >> 2), c);
  if (lane == 0) atomicAdd(acc + 8, e);
}

struct PixelState {
  float T, T_final;
  uint32_t last_contributor;
  float dpix[3];
  float bg_dot_dpixel;
  float accum_rec[3];
  float last_color[3];
  float last_alpha;
};

__device__ __forceinline__ void blend_backward_tile(const TileJob& job, const BlendSource& src, float* grad_acc) {
  __shared__ float4 s_a[kBatch];
  __shared__ float4 s_b[kBatch];
  __shared__ float4 s_c[kBatch];
  __shared__ uint32_t s_g[kBatch];
  __shared__ uint32_t s_warp_last[kBlendWarps];
  const BlendPatch patch = BlendPatch::make(job.tile_x, job.tile_y);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint2 range = job.range;
  const uint32_t n = range.y - range.x;

  const int64_t HW = (int64_t)job.H * job.W;
  PixelState ps[kBlendPx];
  uint32_t thread_last = 0;
#pragma unroll
  for (int i = 0; i < kBlendPx; ++i) {
    PixelState& s = ps[i];
    const bool in = patch.inside(i, job.W, job.H);
    const int64_t pix = in ? patch.pixel(i, job.W) : 0;
    s.T_final = in ? job.final_T[pix] : 0.f;
    s.T = s.T_final;
    s.last_contributor = in ? job.n_contrib[pix] : 0u;
    if (s.last_contributor > n) s.last_contributor = n;
    thread_last = max(thread_last, s.last_contributor);
    s.dpix[0] = in ? job.dL_dpix[pix] : 0.f;
    s.dpix[1] = in ? job.dL_dpix[HW + pix] : 0.f;
    s.dpix[2] = in ? job.dL_dpix[2 * HW + pix] : 0.f;
    s.bg_dot_dpixel = 0.f;
#pragma unroll
    for (int ch = 0; ch < 3; ch++) s.bg_dot_dpixel += job.bg[ch] * s.dpix[ch];
    s.accum_rec[0] = s.accum_rec[1] = s.accum_rec[2] = 0.f;
    s.last_color[0] = s.last_color[1] = s.last_color[2] = 0.f;
    s.last_alpha = 0.f;
  }
  const float ddelx_dx = 0.5 * job.W;
  const float ddely_dy = 0.5 * job.H;

  const uint32_t warp_last = __reduce_max_sync(kFullMask, thread_last);
  if (lane == 0) s_warp_last[warp] = warp_last;
  __syncthreads();
  uint32_t block_last = 0;
#pragma unroll
  for (int w = 0; w < kBlendWarps; ++w) block_last = max(block_last, s_warp_last[w]);

  for (int hi = (int)block_last; hi > 0; hi -= kBatch) {
    const int cnt = min(kBatch, hi);
    __syncthreads();
    stage_batch(src, range.x, hi, cnt, /*reverse=*/true, s_a, s_b, s_c, s_g);
    __syncthreads();
    for (int k = 0; k * 32 < cnt; ++k) {
      const int j = k * 32 + lane;
      bool hit = false;
      if (j < cnt && (uint32_t)(hi - 1 - j) < warp_last) hit = patch.hit(s_a[j], s_b[j]);
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        const uint32_t pos = (uint32_t)(hi - 1 - jj);
        const float4 a = s_a[jj];
        const float4 b = s_b[jj];
        float v[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        bool contrib = false;
#pragma unroll
        for (int i = 0; i < kBlendPx; ++i) {
          PixelState& s = ps[i];
          if (pos >= s.last_contributor) continue;
          const float2 d = {a.x - patch.pxf, a.y - patch.pyf(i)};
          const float power = splat_power(a, b, d);
          if (power > 0.0f) continue;
          const float G = expf(power);
          const float alpha = fminf(0.99f, b.y * G);
          if (alpha < 1.0f / 255.0f) continue;
          contrib = true;
          const float inv_one_minus_alpha = __frcp_rn(1.f - alpha);
          s.T = s.T * inv_one_minus_alpha;
          const float dchannel_dcolor = alpha * s.T;
          const float4 cv = s_c[jj];
          const float col[3] = {cv.x, cv.y, cv.z};
          float dL_dalpha = 0.0f;
#pragma unroll
          for (int ch = 0; ch < 3; ch++) {
            const float c = col[ch];
            s.accum_rec[ch] = s.last_alpha * s.last_color[ch] + (1.f - s.last_alpha) * s.accum_rec[ch];
            s.last_color[ch] = c;
            const float dL_dchannel = s.dpix[ch];
            dL_dalpha += (c - s.accum_rec[ch]) * dL_dchannel;
            v[6 + ch] += dchannel_dcolor * dL_dchannel;
          }
          dL_dalpha *= s.T;
          s.last_alpha = alpha;
          dL_dalpha += (-s.T_final * inv_one_minus_alpha) * s.bg_dot_dpixel;
          const float dL_dG = b.y * dL_dalpha;
          const float gdx = G * d.x;
          const float gdy = G * d.y;
          const float dG_ddelx = -gdx * a.z - gdy * a.w;
          const float dG_ddely = -gdy * b.x - gdx * a.w;
          v[0] += dL_dG * dG_ddelx * ddelx_dx;
          v[1] += dL_dG * dG_ddely * ddely_dy;
          v[2] += -0.5f * gdx * d.x * dL_dG;
          v[3] += -0.5f * gdx * d.y * dL_dG;
          v[4] += -0.5f * gdy * d.y * dL_dG;
          v[5] += G * dL_dalpha;
        }
        const unsigned cm = __ballot_sync(kFullMask, contrib);
        if (cm == 0) continue;
        float* acc = grad_acc + 12 * (size_t)s_g[jj];
        if ((cm & (cm - 1)) == 0) {  // one contributing lane: add its values directly
          if (contrib) {
#pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(acc + q, v[q]);
          }
        } else {
          warp_reduce_add9(v, acc, lane);
        }
      }
    }
  }
}

// One view: block (x, y) back-propagates tile (x, y).
__global__ void __launch_bounds__(kBlendThreads) render_backward_kernel(RenderParams p) {
  TileJob job;
  job.tile_x = blockIdx.x;
  job.tile_y = blockIdx.y;
  job.W = p.W;
  job.H = p.H;
  job.range = checked_range(p.ranges, blockIdx.y * p.gx + blockIdx.x, p.capacity);
  job.bg = p.bg;
  job.out_color = nullptr;
  job.final_T = p.final_T;
  job.n_contrib = p.n_contrib;
  job.dL_dpix = p.dL_dpix;
  blend_backward_tile(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P, p.capacity}, p.grad_acc);
}

// All views of a batch in one launch: block b back-propagates global tile b.
__global__ void __launch_bounds__(kBlendThreads) batch_render_backward_kernel(const __grid_constant__ BatchRenderParams p) {
  const TileJob job = batch_tile_job(p, blockIdx.x);
  blend_backward_tile(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P * (uint32_t)p.V, p.capacity},
                      p.grad_acc);
}

}  // namespace

void launch_render_backward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  render_backward_kernel<<<dim3(p.gx, p.gy), kBlendThreads, 0, s>>>(p);
}

void launch_batch_render_backward(const BatchRenderParams& p, cudaStream_t s) {
  if (p.total_tiles == 0) return;
  batch_render_backward_kernel<<<p.total_tiles, kBlendThreads, 0, s>>>(p);
}

}  // namespace omnigs
