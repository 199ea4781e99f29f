// Backward back-to-front blend of one 16x16 tile per block (backward.cu:672-843).
//
// Per pixel this replays the reference's recurrence: start from the stored final transmittance
// and last-contributor index, walk the tile's instances from the back, undo T /= (1 - alpha) and
// accumulate the colour behind each splat (the reference defers that update to the next splat it
// meets; here it is applied right after the splat, the same sums).  A thread's two pixels share
// their column, so their arithmetic runs in packed f32x2 instructions, lane x for the upper pixel
// and lane y for the lower: one issue slot for both pixels' FMAs.  One approximate reciprocal of
// 1 - alpha serves both of the reference's divisions by it (relative error ~1e-7 per step, far
// inside the gradients' 1e-3 tolerance).  The per-(pixel, splat) gradients (2 screen-space mean,
// 3 conic, 1 opacity, 3 colour) are not pushed with 9 global atomics per pixel as in the
// reference (and the mean terms are summed as w dx and w dy with w = G dL/dalpha, without the
// opacity and the conic, the conic terms without the opacity, all without their constant factors
// -W/2, -H/2, -1/2: the backward preprocess applies those per Gaussian): a thread first sums them
// over its two
// pixels and writes the 9 sums to its warp's shared buffer; every second contributing splat the
// warp that owns the 8 x 8 patch reduces the buffer transposed (one lane per splat and value, 32
// terms each) and adds the accumulator records with one atomic per value.  Warps skip splats
// that cannot reach alpha >= 1/255 in their patch or that lie behind all of their pixels' last
// contributors, and the block starts at the batch holding its largest last contributor instead of
// at the end of the range.
#include "blend_common.cuh"

namespace omnigs {
namespace {

// Per-warp buffer of the lane values of contributing splats: row 9 h + q holds value q of buffered
// splat h for the 32 lanes.  The row stride of 36 floats puts the 16-byte reads of 8 consecutive
// rows (one quarter-warp) on distinct banks; the lanes' writes of one row are consecutive words.
constexpr int kRedStride = 36;

// Adds the buffered splats' lane sums to their accumulator records: lane t sums row t over the
// 32 lanes (eight 16-byte reads, packed adds) and adds the total with one atomic.
__device__ __forceinline__ void flush_reduction(float (*red)[kRedStride], const uint32_t* gidx, int n,
                                                float* grad_acc, int lane) {
  __syncwarp();
  for (int t = lane; t < n * 9; t += 32) {
    const int h = t / 9, q = t - 9 * h;
    const float4* row = reinterpret_cast<const float4*>(red[t]);
    float2 s0 = make_float2(0.f, 0.f), s1 = s0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float4 x = row[i];
      s0 = add2(s0, make_float2(x.x, x.y));
      s1 = add2(s1, make_float2(x.z, x.w));
    }
    s0 = add2(s0, s1);
    atomicAdd(grad_acc + 12 * (size_t)gidx[h] + q, s0.x + s0.y);
  }
  __syncwarp();  // the rows are rewritten next
}

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Eight resident blocks per SM (at most 64 registers per thread) measured fastest on a B200.
constexpr int kBlendBwdMinBlocks = 8;

// kRecompute (transmittance checkpointing): the forward stored no per-pixel state; each pixel's
// final transmittance and last contributor are recomputed first by the forward's own front-to-back
// pass without colour (forward_pass), which yields the values the forward would have stored.
template <int kBatch, bool kWrap, bool kRecompute>
__device__ __forceinline__ void blend_backward_tile(const TileJob& job, const BlendSource& src, float* grad_acc) {
  static_assert(kBlendPx == 2, "the backward blend packs a thread's two pixels into f32x2 lanes");
  __shared__ float4 s_a[kBatch];
  __shared__ float4 s_b[kBatch];
  __shared__ float4 s_c[kBatch];
  __shared__ uint32_t s_g[kBatch];
  __shared__ uint32_t s_warp_last[kBlendWarps];
  // Two buffered splats (18 rows: one flush round) measured fastest on a B200: larger buffers cost
  // occupancy (shared memory, registers) faster than they save reduction instructions.  Storing
  // the values in pairs (five 8-byte stores, two lanes reducing each pair row) measured slower:
  // 1.03 -> 1.12 ms per 1M-Gaussian view.
  constexpr int kRedSplats = 2;
  __shared__ __align__(16) float s_red[kBlendWarps][kRedSplats * 9][kRedStride];
  __shared__ uint32_t s_red_g[kBlendWarps][kRedSplats];
  const BlendPatch patch = BlendPatch::make(job.tile_x, job.tile_y, job.wrap_w);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint2 range = job.range;
  const uint32_t n = range.y - range.x;

  // Per-pixel state of the thread's two pixels, lane x = row py0, lane y = row py0 + 4.
  const int64_t HW = (int64_t)job.H * job.W;
  float Tf[2], dp[3][2];
  uint32_t lc[2];
  if (kRecompute) {
    float2 Tr, c0, c1, c2;
    uint32_t l0, l1;
    forward_pass<kBatch, kWrap, false>(job, src, patch, s_a, s_b, nullptr, Tr, l0, l1, c0, c1, c2);
    Tf[0] = patch.inside(0, job.W, job.H) ? Tr.x : 0.f;
    Tf[1] = patch.inside(1, job.W, job.H) ? Tr.y : 0.f;
    lc[0] = min(l0, n);
    lc[1] = min(l1, n);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const bool in = patch.inside(i, job.W, job.H);
    const int64_t pix = in ? patch.pixel(i, job.W) : 0;
    if (!kRecompute) {
      Tf[i] = in ? job.final_T[pix] : 0.f;
      lc[i] = in ? min(job.n_contrib[pix], n) : 0u;
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) dp[ch][i] = in ? job.dL_dpix[ch * HW + pix] : 0.f;
  }
  const float2 T_final = make_float2(Tf[0], Tf[1]);
  const float2 neg_T_final = make_float2(-Tf[0], -Tf[1]);  // (folded into neg_T_bg below)
  float2 T = T_final;
  const float2 dp0 = make_float2(dp[0][0], dp[0][1]);
  const float2 dp1 = make_float2(dp[1][0], dp[1][1]);
  const float2 dp2 = make_float2(dp[2][0], dp[2][1]);
  float2 bgdot = make_float2(0.f, 0.f);
  bgdot = fma2(f2(job.bg[0]), dp0, bgdot);
  bgdot = fma2(f2(job.bg[1]), dp1, bgdot);
  bgdot = fma2(f2(job.bg[2]), dp2, bgdot);
  const float2 neg_T_bg = mul2(neg_T_final, bgdot);
  // the colour of everything behind the current splat, accumulated back to front, enters the
  // gradients only through its dot product with dL/dpix: that product is accumulated instead
  float2 acc_dp = make_float2(0.f, 0.f);
  const float2 pyf = make_float2(patch.pyf(0), patch.pyf(1));

  float(*red)[kRedStride] = s_red[threadIdx.x >> 5];
  int nred = 0;  // buffered splats (warp-uniform)

  const uint32_t warp_last = __reduce_max_sync(kFullMask, max(lc[0], lc[1]));
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
      // (the branch skips the test for splats behind every last contributor of the warp: evaluating
      // it in every lane measured 3 % slower)
      if (j < cnt && (uint32_t)(hi - 1 - j) < warp_last) hit = patch.template hit<kWrap>(s_a[j], s_b[j]);
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        const uint32_t pos = (uint32_t)(hi - 1 - jj);
        // No per-lane branches: a pixel behind its last contributor, or that this splat does not
        // reach, is inactive through act0 / act1, and the masked alpha = G = 0 makes every one of
        // its 9 values exactly 0.  The two divergent branches measured on a B200 as 7 % of the
        // kernel (1.027 -> 0.955 ms per view; only the inner one removed: 1.088).
        float v[9];
        bool act0 = pos < lc[0], act1 = pos < lc[1];
        {
          const float4 a = s_a[jj];
          const float4 b = s_b[jj];
          const float dx = patch.template center_x<kWrap>(a.x) - patch.pxf;
          const float2 dy = sub2(f2(a.y), pyf);
          const float2 power = splat_power2(a, b, dx, dy);
          const float2 G = make_float2(expf(power.x), expf(power.y));
          const float2 alpha = make_float2(fminf(0.99f, b.y * G.x), fminf(0.99f, b.y * G.y));
          act0 = act0 && !(power.x > 0.0f) && !(alpha.x < 1.0f / 255.0f);
          act1 = act1 && !(power.y > 0.0f) && !(alpha.y < 1.0f / 255.0f);
          // a warp-uniform skip of the gradient arithmetic when no pixel of the warp blends this
          // splat (measured 0.904 -> 0.898 ms per view against testing after the arithmetic)
          if (!__any_sync(kFullMask, act0 || act1)) continue;
          {
            // A pixel this splat does not touch gets alpha = G = 0 and 1 / (1 - alpha) = 1, which
            // leaves its state unchanged and contributes zero to every gradient.
            const float2 ae = make_float2(act0 ? alpha.x : 0.f, act1 ? alpha.y : 0.f);
            const float2 Ge = make_float2(act0 ? G.x : 0.f, act1 ? G.y : 0.f);
            const float2 onem = sub2(f2(1.f), ae);
            const float2 inv = make_float2(act0 ? rcp_approx(onem.x) : 1.f, act1 ? rcp_approx(onem.y) : 1.f);
            T = mul2(T, inv);  // transmittance in front of this splat
            const float2 dcd = mul2(ae, T);
            const float4 cv = s_c[jj];
            // (this splat's colour minus the colour behind it) . dL/dpix; the colour behind becomes
            // alpha c + (1 - alpha) acc, so its product with dL/dpix grows by alpha times this
            float2 c_dp = mul2(f2(cv.x), dp0);
            c_dp = fma2(f2(cv.y), dp1, c_dp);
            c_dp = fma2(f2(cv.z), dp2, c_dp);
            float2 dLda = sub2(c_dp, acc_dp);
            acc_dp = fma2(ae, dLda, acc_dp);
            dLda = mul2(dLda, T);
            dLda = fma2(neg_T_bg, inv, dLda);  // the background term -T_final / (1 - alpha) bg.dL/dpix
            // With q = G dL/dG = o G dL/dalpha and the conic (a, b, c):
            //   dL/d(delta x) = -q (a dx + b dy), dL/d(delta y) = -q (c dy + b dx),
            //   dL/d(conic) = -q (dx^2, dx dy, dy^2) / 2.
            // The per-pixel sums keep only w dx, w dy, w dx^2, ... with w = G dL/dalpha = q / o:
            // the opacity and the conic (constant over the Gaussian's pixels) and the constant
            // factors -W/2, -H/2 and -1/2 are applied once per Gaussian by the backward
            // preprocess.  The thread's two pixels share dx, so the sums over them factor through
            // sum w, sum w dy and sum w dy^2.
            const float2 w5 = mul2(Ge, dLda);
            const float2 q = w5;
            const float2 qy = mul2(q, dy);
            const float qs = q.x + q.y, qdy = qy.x + qy.y;
            v[0] = dx * qs;
            v[1] = qdy;
            v[2] = dx * v[0];
            v[3] = dx * qdy;
            v[4] = fmaf(qy.x, dy.x, qy.y * dy.y);
            v[5] = w5.x + w5.y;
            v[6] = fmaf(dcd.x, dp0.x, dcd.y * dp0.y);
            v[7] = fmaf(dcd.x, dp1.x, dcd.y * dp1.y);
            v[8] = fmaf(dcd.x, dp2.x, dcd.y * dp2.y);
          }
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) red[nred * 9 + q][lane] = v[q];
        if (lane == 0) s_red_g[warp][nred] = s_g[jj];
        if (++nred == kRedSplats) {
          flush_reduction(red, s_red_g[warp], nred, grad_acc, lane);
          nred = 0;
        }
      }
    }
  }
  if (nred) flush_reduction(red, s_red_g[warp], nred, grad_acc, lane);
}

// One view: block (x, y) back-propagates tile (x, y).
template <int kBatch, bool kRecompute>
__global__ void __launch_bounds__(kBlendThreads, kBlendBwdMinBlocks) render_backward_kernel(RenderParams p) {
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
  job.wrap_w = 0.f;
  blend_backward_tile<kBatch, false, kRecompute>(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P, p.capacity},
                                                 p.grad_acc);
}

// All views of a batch in one launch: block b back-propagates global tile b.
template <int kBatch, bool kWrap>
__global__ void __launch_bounds__(kBlendThreads, kBlendBwdMinBlocks) batch_render_backward_kernel(const __grid_constant__ BatchRenderParams p) {
  const TileJob job = batch_tile_job(p, blockIdx.x);
  blend_backward_tile<kBatch, kWrap, false>(job, BlendSource{p.point_list, p.splat, p.color, (uint32_t)p.P * (uint32_t)p.V, p.capacity},
                                            p.grad_acc);
}

template <bool kWrap>
void launch_batch_blend(const BatchRenderParams& p, cudaStream_t s) {
  switch (blend_batch_size(true)) {
    case 128: batch_render_backward_kernel<128, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
    case 512: batch_render_backward_kernel<512, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
    default: batch_render_backward_kernel<256, kWrap><<<p.total_tiles, kBlendThreads, 0, s>>>(p); break;
  }
}

template <bool kRecompute>
void launch_single_view_backward(const RenderParams& p, const dim3 grid, cudaStream_t s) {
  switch (blend_batch_size(true)) {
    case 128: render_backward_kernel<128, kRecompute><<<grid, kBlendThreads, 0, s>>>(p); break;
    case 512: render_backward_kernel<512, kRecompute><<<grid, kBlendThreads, 0, s>>>(p); break;
    default: render_backward_kernel<256, kRecompute><<<grid, kBlendThreads, 0, s>>>(p); break;
  }
}

}  // namespace

void launch_render_backward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  const dim3 grid(p.gx, p.gy);
  if (p.final_T == nullptr)  // transmittance checkpointing: recompute the per-pixel state
    launch_single_view_backward<true>(p, grid, s);
  else
    launch_single_view_backward<false>(p, grid, s);
}

void launch_batch_render_backward(const BatchRenderParams& p, cudaStream_t s) {
  if (p.total_tiles == 0) return;
  if (p.seam_wrap)
    launch_batch_blend<true>(p, s);
  else
    launch_batch_blend<false>(p, s);
}

}  // namespace omnigs
