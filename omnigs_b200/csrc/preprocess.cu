// Forward preprocess of lonlat splats, one thread per Gaussian.
//
// Evaluates the reference's FP32 sequence (forward.cu:592-703): near cull at r^2 <= 0.04,
// equirect projection, 3D and 2D covariance, conic, radius, clamped tile rect and SH colour.
// Outputs per Gaussian: radius, the 32-byte splat record and colour record read by the blend
// kernels, the radial depth (+inf for culled Gaussians: it is the depth-sort key of the binning)
// and tiles_touched; the instance total is summed on the device (block reduction + one atomic
// per block), so nothing is copied to the host (the reference copies num_rendered back between
// its scan and its duplication, rasterizer_impl.cu:622-628).
//
// Besides the reference's outputs, each visible splat gets the half-extents of the axis-aligned
// box outside which its alpha is provably below 1/255; the blend kernels use them to skip a splat
// for a whole warp without changing any per-pixel decision.
#include "device_util.cuh"
#include "kernels.h"
#include "lonlat_math.cuh"

namespace omnigs {
namespace {

// Half-extents (pixels) of the box that contains every pixel where o * exp(power) can reach the
// reference's 1/255 skip threshold (forward.cu:436-438).  power = -d^T Q d / 2 with Q the conic,
// so alpha >= 1/255 needs d^T Q d <= 2 tau, tau = ln(255 o) (+0.01 slack for expf error and FP32
// rounding of `power`).  The ellipse's x half-extent is sqrt(2 tau (Q^-1)_xx).  Non-finite inputs
// or an indefinite conic disable culling (+inf); an opacity that can never reach 1/255 culls
// everywhere (-inf).
__device__ __forceinline__ float2 cull_half_extent(float a, float b, float c, float o) {
  const float inf = __int_as_float(0x7f800000);
  if (!(isfinite(a) && isfinite(b) && isfinite(c) && isfinite(o))) return make_float2(inf, inf);
  if (!(o > 0.0f)) return make_float2(-inf, -inf);
  const double tau = log(255.0 * (double)o) + 0.01;
  if (tau <= 0.0) return make_float2(-inf, -inf);
  const double A = a, B = b, C = c;
  const double det = A * C - B * B;
  if (!(A > 0.0) || !(det > 0.0)) return make_float2(inf, inf);
  const double hx = sqrt(2.0 * tau * C / det) * (1.0 + 1e-4) + 1e-2;
  const double hy = sqrt(2.0 * tau * A / det) * (1.0 + 1e-4) + 1e-2;
  return make_float2(__double2float_ru(hx), __double2float_ru(hy));
}

__global__ void __launch_bounds__(kScanBlock) preprocess_kernel(PreprocessParams p) {
  __shared__ uint32_t s_warp[kScanBlock / 32];
  const int idx = blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  uint32_t touched = 0;
  if (idx < p.P) {
    p.radii[idx] = 0;
    float depth_key = __int_as_float(0x7f800000);  // culled Gaussians sort last
    const float* vm = p.viewmatrix;
    const float3 p_orig = {p.means3D[3 * idx], p.means3D[3 * idx + 1], p.means3D[3 * idx + 2]};
    // near cull, auxiliary.h:198-220 (no frustum test for lonlat)
    const float3 p_view = xform_point(p_orig, vm);
    const float rr = p_view.x * p_view.x + p_view.y * p_view.y + p_view.z * p_view.z;
    if (!(rr <= 0.04f)) {
      const float r = sqrtf(rr);
      // point3ToLonlatScreen, auxiliary.h:236-248
      const float inv_r = 1.0f / (r + 0.0000001f);
      const float lon = atan2f(p_view.x, p_view.z);
      const float lat = asinf(p_view.y * inv_r);
      const float scr_x = lon * kInvPi;
      const float scr_y = lat * kTwoInvPi;
      float cov3D[6];
      if (p.cov3D_precomp != nullptr) {
#pragma unroll
        for (int k = 0; k < 6; ++k) cov3D[k] = p.cov3D_precomp[6 * idx + k];
      } else {
        const float3 s = {p.scales[3 * idx], p.scales[3 * idx + 1], p.scales[3 * idx + 2]};
        const float4 q = {p.rotations[4 * idx], p.rotations[4 * idx + 1], p.rotations[4 * idx + 2],
                          p.rotations[4 * idx + 3]};
        cov3d_from_scale_rot(s, p.scale_modifier, q, cov3D);
        // The reference stores cov3D to global memory here (forward.cu:650), so its 2D-covariance
        // code reloads the view matrix and recomputes the camera-space mean instead of reusing
        // the values above.  This compiler barrier keeps the same dataflow (and therefore the
        // same FMA contraction) so radii and tile rects stay bit-identical.
        asm volatile("" ::: "memory");
      }
      const float3 cov = cov2d_lonlat(p_orig, p.W, p.H, cov3D, vm);
      const float det = (cov.x * cov.z - cov.y * cov.y);
      if (det != 0.0f) {
        const float det_inv = 1.f / det;
        const float3 conic = {cov.z * det_inv, -cov.y * det_inv, cov.x * det_inv};
        const float mid = 0.5f * (cov.x + cov.z);
        const float lambda1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
        const float lambda2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
        const float my_radius = ceilf(3.f * sqrtf(fmaxf(lambda1, lambda2)));
        const float2 point_image = {ndc_to_pixel(scr_x, p.W), ndc_to_pixel(scr_y, p.H)};
        const int radius = (int)my_radius;
        int2 rmin, rmax;
        tile_rect(point_image, radius, p.gx, p.gy, rmin, rmax);
        const uint32_t area = (uint32_t)(rmax.x - rmin.x) * (uint32_t)(rmax.y - rmin.y);
        if (area != 0) {
          float4 col;
          if (p.colors_precomp == nullptr) {
            const float* shg = p.shs + (size_t)idx * p.M * 3;
            auto sh = [shg](int k) { return v3(__ldg(shg + 3 * k), __ldg(shg + 3 * k + 1), __ldg(shg + 3 * k + 2)); };
            const V3 pos = v3(p_orig.x, p_orig.y, p_orig.z);
            const V3 cam = v3(p.campos[0], p.campos[1], p.campos[2]);
            const V3 c = sh_color_unclamped(p.D, pos, cam, sh);
            const uint32_t bits = (c.x < 0 ? 1u : 0u) | (c.y < 0 ? 2u : 0u) | (c.z < 0 ? 4u : 0u);
            col = make_float4(clamp_at_zero(c.x), clamp_at_zero(c.y), clamp_at_zero(c.z),
                              __uint_as_float(bits));
          } else {
            col = make_float4(p.colors_precomp[3 * idx], p.colors_precomp[3 * idx + 1],
                              p.colors_precomp[3 * idx + 2], __uint_as_float(0u));
          }
          const float opacity = p.opacities[idx];
          const float2 ext = cull_half_extent(conic.x, conic.y, conic.z, opacity);
          p.splat[2 * idx] = make_float4(point_image.x, point_image.y, conic.x, conic.y);
          p.splat[2 * idx + 1] = make_float4(conic.z, opacity, ext.x, ext.y);
          p.color[idx] = col;
          depth_key = r;
          p.radii[idx] = radius;
          const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
          p.grad_acc[3 * idx] = z4;
          p.grad_acc[3 * idx + 1] = z4;
          p.grad_acc[3 * idx + 2] = z4;
          touched = area;
        }
      }
    }
    p.depth[idx] = depth_key;
    p.tiles_touched[idx] = touched;
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
    for (int w = 0; w < kScanBlock / 32; ++w) total += s_warp[w];
    if (total) atomicAdd(&p.hdr->num_rendered64, total);
  }
}

}  // namespace

void launch_preprocess(const PreprocessParams& p, cudaStream_t s) {
  if (p.P <= 0) return;
  const int blocks = (p.P + kScanBlock - 1) / kScanBlock;
  preprocess_kernel<<<blocks, kScanBlock, 0, s>>>(p);
}

}  // namespace omnigs
