// Backward back-to-front blend of one 16x16 tile per block (backward.cu:672-843).
//
// Per pixel this replays the reference's recurrence exactly: start from the stored final
// transmittance and last-contributor index, walk the tile's instances from the back, undo
// T /= (1 - alpha) and accumulate the colour-behind term.  The per-(pixel, splat) gradients
// (2 screen-space mean, 3 conic, 1 opacity, 3 colour) are not pushed with 9 global atomics per
// pixel as in the reference: the warp that owns an 8x4 pixel patch reduces them first, with a
// reduce-scatter of 8 values (9 shuffles) plus a butterfly for the ninth, and then 8 lanes add one
// 32-byte accumulator record per splat.  Warps skip splats whose alpha-support box misses their
// patch or that lie behind all of their pixels' last contributors, and the block starts at the
// batch holding its largest last contributor instead of at the end of the range.
#include "device_util.cuh"
#include "kernels.h"

namespace omnigs {
namespace {

constexpr int kBatch = 256;

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

__global__ void __launch_bounds__(256) render_backward_kernel(RenderParams p) {
  __shared__ float4 s_a[kBatch];
  __shared__ float4 s_b[kBatch];
  __shared__ float4 s_c[kBatch];
  __shared__ uint32_t s_g[kBatch];
  __shared__ uint32_t s_warp_last[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wx0 = blockIdx.x * 16 + (warp & 1) * 8;
  const int wy0 = blockIdx.y * 16 + (warp >> 1) * 4;
  const int px = wx0 + (lane & 7), py = wy0 + (lane >> 3);
  const bool inside = px < p.W && py < p.H;
  const float2 pixf = {(float)px, (float)py};
  const float wcx = (float)wx0 + 3.5f, wcy = (float)wy0 + 1.5f;

  uint2 range = p.ranges[blockIdx.y * p.gx + blockIdx.x];
  if (range.y > (uint64_t)p.capacity || range.x > range.y) range = make_uint2(0, 0);
  const uint32_t n = range.y - range.x;

  const int64_t pix = (int64_t)py * p.W + px;
  const int64_t HW = (int64_t)p.H * p.W;
  const float T_final = inside ? p.final_T[pix] : 0.f;
  float T = T_final;
  uint32_t last_contributor = inside ? p.n_contrib[pix] : 0u;
  if (last_contributor > n) last_contributor = n;
  float dpix[3] = {0.f, 0.f, 0.f};
  if (inside) {
    dpix[0] = p.dL_dpix[pix];
    dpix[1] = p.dL_dpix[HW + pix];
    dpix[2] = p.dL_dpix[2 * HW + pix];
  }
  float bg_dot_dpixel = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) bg_dot_dpixel += p.bg[i] * dpix[i];
  const float ddelx_dx = 0.5 * p.W;
  const float ddely_dy = 0.5 * p.H;
  float accum_rec[3] = {0.f, 0.f, 0.f};
  float last_color[3] = {0.f, 0.f, 0.f};
  float last_alpha = 0.f;

  const uint32_t warp_last = __reduce_max_sync(kFullMask, last_contributor);
  if (lane == 0) s_warp_last[warp] = warp_last;
  __syncthreads();
  uint32_t block_last = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) block_last = max(block_last, s_warp_last[w]);

  for (int hi = (int)block_last; hi > 0; hi -= kBatch) {
    const int cnt = min(kBatch, hi);
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
      const uint32_t pos = (uint32_t)(hi - 1 - (int)threadIdx.x);
      const uint32_t g = p.point_list[range.x + pos];
      if (g < (uint32_t)p.P) {
        s_g[threadIdx.x] = g;
        s_a[threadIdx.x] = p.splat[2 * g];
        s_b[threadIdx.x] = p.splat[2 * g + 1];
        s_c[threadIdx.x] = p.color[g];
      } else {  // unreachable for a consistent instance list; stage a splat that never contributes
        s_g[threadIdx.x] = 0;
        s_a[threadIdx.x] = make_float4(__int_as_float(0x7f800000), 0.f, 0.f, 0.f);
        s_b[threadIdx.x] = make_float4(0.f, 0.f, -__int_as_float(0x7f800000), -__int_as_float(0x7f800000));
        s_c[threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    __syncthreads();
    for (int k = 0; k * 32 < cnt; ++k) {
      const int j = k * 32 + lane;
      bool hit = false;
      if (j < cnt && (uint32_t)(hi - 1 - j) < warp_last) {
        const float4 a = s_a[j];
        const float4 b = s_b[j];
        hit = !(fabsf(a.x - wcx) > b.z + 3.5f || fabsf(a.y - wcy) > b.w + 1.5f);
      }
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        const uint32_t pos = (uint32_t)(hi - 1 - jj);
        float v[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        bool contrib = false;
        if (pos < last_contributor) {
          const float4 a = s_a[jj];
          const float4 b = s_b[jj];
          const float2 d = {a.x - pixf.x, a.y - pixf.y};
          const float power = -0.5f * (a.z * d.x * d.x + b.x * d.y * d.y) - a.w * d.x * d.y;
          if (!(power > 0.0f)) {
            const float G = expf(power);
            const float alpha = fminf(0.99f, b.y * G);
            if (!(alpha < 1.0f / 255.0f)) {
              contrib = true;
              T = T / (1.f - alpha);
              const float dchannel_dcolor = alpha * T;
              const float4 cv = s_c[jj];
              const float col[3] = {cv.x, cv.y, cv.z};
              float dL_dalpha = 0.0f;
#pragma unroll
              for (int ch = 0; ch < 3; ch++) {
                const float c = col[ch];
                accum_rec[ch] = last_alpha * last_color[ch] + (1.f - last_alpha) * accum_rec[ch];
                last_color[ch] = c;
                const float dL_dchannel = dpix[ch];
                dL_dalpha += (c - accum_rec[ch]) * dL_dchannel;
                v[6 + ch] = dchannel_dcolor * dL_dchannel;
              }
              dL_dalpha *= T;
              last_alpha = alpha;
              dL_dalpha += (-T_final / (1.f - alpha)) * bg_dot_dpixel;
              const float dL_dG = b.y * dL_dalpha;
              const float gdx = G * d.x;
              const float gdy = G * d.y;
              const float dG_ddelx = -gdx * a.z - gdy * a.w;
              const float dG_ddely = -gdy * b.x - gdx * a.w;
              v[0] = dL_dG * dG_ddelx * ddelx_dx;
              v[1] = dL_dG * dG_ddely * ddely_dy;
              v[2] = -0.5f * gdx * d.x * dL_dG;
              v[3] = -0.5f * gdx * d.y * dL_dG;
              v[4] = -0.5f * gdy * d.y * dL_dG;
              v[5] = G * dL_dalpha;
            }
          }
        }
        if (__any_sync(kFullMask, contrib)) warp_reduce_add9(v, p.grad_acc + 12 * (size_t)s_g[jj], lane);
      }
    }
  }
}

}  // namespace

void launch_render_backward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  render_backward_kernel<<<dim3(p.gx, p.gy), 256, 0, s>>>(p);
}

}  // namespace omnigs
