// Forward front-to-back alpha blend of one 16x16 tile per block (forward.cu:346-467).
//
// Every pixel evaluates exactly the reference's per-pair arithmetic and control flow (power,
// alpha = min(0.99, o exp(power)), the 1/255 skip, the T < 1e-4 stop), so the image, final
// transmittance and last-contributor index are identical for the same sorted instance list.
// What changes is the work around it:
//  * the 256 threads are 8 warps of 8x4 pixels; for each staged batch a warp ballots which splats'
//    alpha-support boxes (computed in the preprocess) touch its 8x4 footprint and iterates only
//    over those, so pairs that the reference rejects pixel by pixel are skipped a warp at a time;
//  * a warp stops as soon as all of its pixels are saturated (warp vote), and the block stops when
//    every warp has (block vote), as in the reference;
//  * splat geometry and colour are staged together (three float4 per instance) so the inner loop
//    reads only shared memory.
#include "device_util.cuh"
#include "kernels.h"

namespace omnigs {
namespace {

constexpr int kBatch = 256;

__global__ void __launch_bounds__(256) render_forward_kernel(RenderParams p) {
  __shared__ float4 s_a[kBatch];  // x, y, conic a, conic b
  __shared__ float4 s_b[kBatch];  // conic c, opacity, cull half-width, cull half-height
  __shared__ float4 s_c[kBatch];  // r, g, b, clamp bits
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wx0 = blockIdx.x * 16 + (warp & 1) * 8;
  const int wy0 = blockIdx.y * 16 + (warp >> 1) * 4;
  const int px = wx0 + (lane & 7), py = wy0 + (lane >> 3);
  const bool inside = px < p.W && py < p.H;
  const float2 pixf = {(float)px, (float)py};
  const float wcx = (float)wx0 + 3.5f, wcy = (float)wy0 + 1.5f;

  uint2 range = p.ranges[blockIdx.y * p.gx + blockIdx.x];
  if (range.y > (uint64_t)p.capacity || range.x > range.y) range = make_uint2(0, 0);
  const int n = (int)(range.y - range.x);

  bool done = !inside;
  float T = 1.0f;
  float C0 = 0.f, C1 = 0.f, C2 = 0.f;
  uint32_t last_contributor = 0;

  for (int base = 0; base < n; base += kBatch) {
    if (__syncthreads_and(done)) break;
    const int i = base + threadIdx.x;
    if (i < n) {
      const uint32_t g = p.point_list[range.x + i];
      if (g < (uint32_t)p.P) {
        s_a[threadIdx.x] = p.splat[2 * g];
        s_b[threadIdx.x] = p.splat[2 * g + 1];
        s_c[threadIdx.x] = p.color[g];
      } else {  // unreachable for a consistent instance list; stage a splat that never contributes
        s_a[threadIdx.x] = make_float4(__int_as_float(0x7f800000), 0.f, 0.f, 0.f);
        s_b[threadIdx.x] = make_float4(0.f, 0.f, -__int_as_float(0x7f800000), -__int_as_float(0x7f800000));
        s_c[threadIdx.x] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    __syncthreads();
    const int cnt = min(kBatch, n - base);
    bool warp_done = __all_sync(kFullMask, done);
    for (int k = 0; k * 32 < cnt && !warp_done; ++k) {
      const int j = k * 32 + lane;
      bool hit = false;
      if (j < cnt) {
        const float4 a = s_a[j];
        const float4 b = s_b[j];
        hit = !(fabsf(a.x - wcx) > b.z + 3.5f || fabsf(a.y - wcy) > b.w + 1.5f);
      }
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        if (!done) {
          const float4 a = s_a[jj];
          const float4 b = s_b[jj];
          const float2 d = {a.x - pixf.x, a.y - pixf.y};
          const float power = -0.5f * (a.z * d.x * d.x + b.x * d.y * d.y) - a.w * d.x * d.y;
          if (!(power > 0.0f)) {
            const float alpha = fminf(0.99f, b.y * expf(power));
            if (!(alpha < 1.0f / 255.0f)) {
              const float test_T = T * (1 - alpha);
              if (test_T < 0.0001f) {
                done = true;
              } else {
                const float4 c = s_c[jj];
                C0 += c.x * alpha * T;
                C1 += c.y * alpha * T;
                C2 += c.z * alpha * T;
                T = test_T;
                last_contributor = (uint32_t)(base + jj + 1);
              }
            }
          }
        }
        if (__all_sync(kFullMask, done)) {
          warp_done = true;
          break;
        }
      }
    }
  }

  if (inside) {
    const int64_t pix = (int64_t)py * p.W + px;
    const int64_t HW = (int64_t)p.H * p.W;
    p.final_T[pix] = T;
    p.n_contrib[pix] = last_contributor;
    p.out_color[pix] = C0 + T * p.bg[0];
    p.out_color[HW + pix] = C1 + T * p.bg[1];
    p.out_color[2 * HW + pix] = C2 + T * p.bg[2];
  }
}

}  // namespace

void launch_render_forward(const RenderParams& p, cudaStream_t s) {
  if (p.gx <= 0 || p.gy <= 0) return;
  render_forward_kernel<<<dim3(p.gx, p.gy), 256, 0, s>>>(p);
}

}  // namespace omnigs
