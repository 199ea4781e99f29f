// Shared pieces of the forward and backward tile blends: the pixel patch a warp owns, the
// alpha-support test of a splat against it, and the staging of a batch of splats into shared memory.
#pragma once

#include "device_util.cuh"
#include "kernels.h"

namespace omnigs {

// Pixels per thread: a thread owns kBlendPx pixels of one column, 4 rows apart, so a warp (8
// columns x 4 rows of threads) owns an 8 x (4 kBlendPx) patch and a block of kBlendThreads
// threads one 16x16 tile.
#ifndef OMNIGS_BLEND_PX
#define OMNIGS_BLEND_PX 2
#endif
constexpr int kBlendPx = OMNIGS_BLEND_PX;
static_assert(kBlendPx == 1 || kBlendPx == 2 || kBlendPx == 4, "a 16x16 tile splits into 8/kBlendPx warps");
constexpr int kBlendThreads = 256 / kBlendPx;
constexpr int kBlendWarps = kBlendThreads / 32;

// One 16x16 tile of one view, as a blend block sees it.  The per-pixel pointers are the view's.
struct TileJob {
  int tile_x, tile_y;
  int W, H;
  uint2 range;              // [begin, end) of the tile's instances in the sorted list
  const float* bg;          // [3]
  float* out_color;         // [3,H,W]
  float* final_T;           // [H*W]
  uint32_t* n_contrib;      // [H*W]
  const float* dL_dpix;     // [3,H,W] (backward)
  float wrap_w;             // image width when blending across the longitude seam, else 0
};

// The sorted instance list and the per-record splat data it points into.
struct BlendSource {
  const uint32_t* point_list;  // record index per instance
  const float4* splat;         // [records][2]
  const float4* color;         // [records]
  uint32_t num_records;
  int64_t capacity;            // instances the list can hold; larger range bounds are rejected
};

// Tile range read from the ranges table, emptied if inconsistent with the list's capacity.
__device__ __forceinline__ uint2 checked_range(const uint2* ranges, uint32_t tile, int64_t capacity) {
  uint2 range = ranges[tile];
  if (range.y > (uint64_t)capacity || range.x > range.y) range = make_uint2(0, 0);
  return range;
}

// Rows of the patch a warp owns (8 columns wide).
constexpr int kPatchRows = 4 * kBlendPx;

struct BlendPatch {
  int px, py0;       // this thread's column and first row
  float pxf;         // column as float
  float wx0, wy0;    // first column and row of the warp's patch
  float wcx;         // centre column of the warp's patch
  float wrap_w;      // image width in seam-wrapping mode, else 0

  // x of the splat's copy (shifted by a multiple of the image width) nearest this patch; the
  // splat's own x unless the seam wraps (kWrap, a template flag so that the non-wrapping kernels
  // carry no trace of it).
  template <bool kWrap>
  __device__ __forceinline__ float center_x(float ax) const {
    return kWrap ? ax - wrap_w * rintf((ax - wcx) / wrap_w) : ax;
  }

  static __device__ __forceinline__ BlendPatch make(int tile_x, int tile_y, float wrap_w = 0.f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wx0 = tile_x * 16 + (warp & 1) * 8;
    const int wy0 = tile_y * 16 + (warp >> 1) * kPatchRows;
    BlendPatch b;
    b.px = wx0 + (lane & 7);
    b.py0 = wy0 + (lane >> 3);
    b.pxf = (float)b.px;
    b.wx0 = (float)wx0;
    b.wy0 = (float)wy0;
    b.wcx = (float)wx0 + 3.5f;
    b.wrap_w = wrap_w;
    return b;
  }
  __device__ __forceinline__ int py(int i) const { return py0 + 4 * i; }
  __device__ __forceinline__ float pyf(int i) const { return (float)(py0 + 4 * i); }
  __device__ __forceinline__ bool inside(int i, int W, int H) const { return px < W && py(i) < H; }
  __device__ __forceinline__ int64_t pixel(int i, int W) const { return (int64_t)py(i) * W + px; }

  // Whether the splat (a = {x, y, conic a, conic b}, b = {conic c, opacity, thr, det}) can reach
  // alpha >= 1/255 at some pixel centre of the patch: the minimum of its quadratic form
  // q(d) = a dx^2 + 2 b dx dy + c dy^2 over the patch's offsets d = centre - pixel, a rectangle
  // [dxl, dxh] x [dyl, dyh], against thr.  A convex form's minimum over a rectangle that does not
  // contain its centre lies on a side facing the centre (KKT), so two candidate sides suffice: the
  // column side at dxn (the x offset nearest 0) minimised over dy, and the row side at dyn minimised
  // over dx.  Scaled by c (resp. a) each is a clamp and a sum of squares without division:
  //   c q(dxn, dy) = (c dy + b dxn)^2 + det dxn^2, minimised at c dy = clamp(-b dxn, c dyl, c dyh).
  // When the centre lies inside the patch both offsets are 0 and the value is 0.  Any other side
  // value is q at a point of the patch, so it never claims a miss wrongly.  Written as a negated
  // "misses" test so that NaN (det of a non-positive-definite conic, non-finite inputs) hits: the
  // per-pixel test decides.
  template <bool kWrap>
  __device__ __forceinline__ bool hit(const float4& a, const float4& b) const {
    const float dxh = center_x<kWrap>(a.x) - wx0, dxl = dxh - 7.0f;
    const float dyh = a.y - wy0, dyl = dyh - (float)(kPatchRows - 1);
    const float dxn = fminf(fmaxf(dxl, 0.0f), dxh), dyn = fminf(fmaxf(dyl, 0.0f), dyh);
    const float bx = a.w * dxn, by = a.w * dyn;
    const float sx = fminf(fmaxf(-bx, b.x * dyl), b.x * dyh) + bx;
    const float sy = fminf(fmaxf(-by, a.z * dxl), a.z * dxh) + by;
    const float vx = fmaf(sx, sx, b.w * dxn * dxn);
    const float vy = fmaf(sy, sy, b.w * dyn * dyn);
    return !(vx > b.x * b.z && vy > a.z * b.z);
  }
};

// Exponent of the splat's Gaussian at offset d = centre - pixel (forward.cu:416, backward.cu:763):
//   power = -0.5 (ca dx^2 + cc dy^2) - cb dx dy.
// The reference leaves the rounding of this expression to the compiler's FMA contraction.  It is
// written here with explicit roundings in the one fusion that reproduces the reference's compiled
// results bit for bit (checked on the 1M-Gaussian 2048x1024 scene: identical transmittance, last
// contributors and image): ca dx dx fused into the sum with the rounded cc dy dy, the cb dx dy term
// rounded on its own.  Being explicit keeps the result independent of how the surrounding kernel is
// structured (a thread owning several pixels lets the compiler share products between them and
// choose other fusions).  The forward and backward use the same function, so they agree on every
// 1/255 and saturation decision.
__device__ __forceinline__ float splat_power(const float4& a, const float4& b, float2 d) {
  const float ca_dx = __fmul_rn(a.z, d.x), cc_dy = __fmul_rn(b.x, d.y), cb_dx = __fmul_rn(a.w, d.x);
  const float quad = __fmaf_rn(ca_dx, d.x, __fmul_rn(cc_dy, d.y));
  return __fsub_rn(__fmul_rn(-0.5f, quad), __fmul_rn(cb_dx, d.y));
}

// Packed f32x2 arithmetic (one instruction for both lanes, each rounded as its scalar form).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// splat_power for two pixels of one column (offsets (dx, dy.x) and (dx, dy.y)), lane by lane
// bit-identical to splat_power.
__device__ __forceinline__ float2 splat_power2(const float4& a, const float4& b, float dx, float2 dy) {
  const float ca_dx = __fmul_rn(a.z, dx), cb_dx = __fmul_rn(a.w, dx);
  const float2 cc_dy = mul2(f2(b.x), dy);
  const float2 quad = fma2(f2(ca_dx), f2(dx), mul2(cc_dy, dy));
  return sub2(mul2(f2(-0.5f), quad), mul2(f2(cb_dx), dy));
}

// Stages instances [base, base + cnt) of the tile's list (from the back when reverse: slot t holds
// position base_hi - 1 - t, with base the exclusive upper end) into shared memory; the colour (s_c)
// only with kColor, the record index only when s_g is not NULL.
template <bool kColor = true>
__device__ __forceinline__ void stage_batch(const BlendSource& src, uint32_t range_begin, int base, int cnt,
                                            bool reverse, float4* s_a, float4* s_b, float4* s_c,
                                            uint32_t* s_g) {
  for (int t = threadIdx.x; t < cnt; t += kBlendThreads) {
    const uint32_t pos = reverse ? (uint32_t)(base - 1 - t) : (uint32_t)(base + t);
    const uint32_t g = src.point_list[range_begin + pos];
    if (g < src.num_records) {
      if (s_g) s_g[t] = g;
      s_a[t] = src.splat[2 * g];
      s_b[t] = src.splat[2 * g + 1];
      if (kColor) s_c[t] = src.color[g];
    } else {  // unreachable for a consistent instance list; stage a splat that never contributes:
              // finite, unit conic, threshold -inf (no patch test hits), opacity 0 (alpha 0)
      if (s_g) s_g[t] = 0;
      s_a[t] = make_float4(0.f, 0.f, 1.f, 0.f);
      s_b[t] = make_float4(1.f, 0.f, -__int_as_float(0x7f800000), 1.f);
      if (kColor) s_c[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

// The forward's front-to-back pass over a tile's instances (forward.cu:394-456) for the thread's two
// pixels (lane x: row py0, lane y: row py0 + 4): transmittance T and last contributor lc, and with
// kColor the blended colour C.  Every pixel evaluates the reference's per-pair arithmetic and control
// flow (power, alpha = min(0.99, o exp(power)), the 1/255 skip, the T < 1e-4 stop), so T and lc are
// the same whether or not colour is blended: the forward kernel runs it with colour, the backward
// runs it without to recompute the state it did not store.  The staging arrays hold kBatch splats.
// The block's threads must all call it (it synchronises the block).
template <int kBatch, bool kWrap, bool kColor>
__device__ __forceinline__ void forward_pass(const TileJob& job, const BlendSource& src, const BlendPatch& patch,
                                             float4* s_a, float4* s_b, float4* s_c, float2& T, uint32_t& lc0,
                                             uint32_t& lc1, float2& C0, float2& C1, float2& C2) {
  static_assert(kBlendPx == 2, "the blend packs a thread's two pixels into f32x2 lanes");
  const int lane = threadIdx.x & 31;
  const uint2 range = job.range;
  const int n = (int)(range.y - range.x);
  bool done0 = !patch.inside(0, job.W, job.H), done1 = !patch.inside(1, job.W, job.H);
  T = f2(1.0f);
  C0 = C1 = C2 = f2(0.f);
  lc0 = lc1 = 0;
  const float2 pyf = make_float2(patch.pyf(0), patch.pyf(1));

  for (int base = 0; base < n; base += kBatch) {
    if (__syncthreads_and(done0 && done1)) break;
    stage_batch<kColor>(src, range.x, base, min(kBatch, n - base), /*reverse=*/false, s_a, s_b, s_c, nullptr);
    __syncthreads();
    const int cnt = min(kBatch, n - base);
    bool warp_done = __all_sync(kFullMask, done0 && done1);
    for (int k = 0; k * 32 < cnt && !warp_done; ++k) {
      const int j = k * 32 + lane;
      // evaluated by every lane (slots past cnt hold stale or unset data, which j < cnt drops):
      // measured 2 % faster than a branch around the test
      const bool hit = patch.template hit<kWrap>(s_a[j], s_b[j]) && j < cnt;
      unsigned m = __ballot_sync(kFullMask, hit);
      while (m) {
        const int jj = k * 32 + __ffs(m) - 1;
        m &= m - 1;
        // No per-lane branches: a pixel that is done, or that this splat does not reach, is
        // inactive through act0 / act1 and its state is updated by selects (alpha 0 adds exactly
        // 0 to the colour).  The divergent branches measured on a B200 as 13 % of the forward
        // (0.614 -> 0.545 ms per view without the one around the pair, 0.532 without both).
        {
          const float4 a = s_a[jj];
          const float4 b = s_b[jj];
          const float dx = patch.template center_x<kWrap>(a.x) - patch.pxf;
          const float2 dy = sub2(f2(a.y), pyf);
          const float2 power = splat_power2(a, b, dx, dy);
          const float2 alpha = make_float2(fminf(0.99f, b.y * expf(power.x)), fminf(0.99f, b.y * expf(power.y)));
          bool act0 = !done0 && !(power.x > 0.0f) && !(alpha.x < 1.0f / 255.0f);
          bool act1 = !done1 && !(power.y > 0.0f) && !(alpha.y < 1.0f / 255.0f);
          {
            const float2 test_T = mul2(T, sub2(f2(1.0f), alpha));
            // a pixel whose transmittance would fall below 1e-4 stops without this splat
            if (act0 && test_T.x < 0.0001f) {
              done0 = true;
              act0 = false;
            }
            if (act1 && test_T.y < 0.0001f) {
              done1 = true;
              act1 = false;
            }
            if (kColor) {
              const float2 ae = make_float2(act0 ? alpha.x : 0.f, act1 ? alpha.y : 0.f);
              const float4 c = s_c[jj];
              // C += colour * alpha * T, rounded as the reference's compiled blend (fused add);
              // a pixel without this splat adds exactly 0
              C0 = fma2(mul2(f2(c.x), ae), T, C0);
              C1 = fma2(mul2(f2(c.y), ae), T, C1);
              C2 = fma2(mul2(f2(c.z), ae), T, C2);
            }
            T = make_float2(act0 ? test_T.x : T.x, act1 ? test_T.y : T.y);
            const uint32_t idx = (uint32_t)(base + jj + 1);
            lc0 = act0 ? idx : lc0;
            lc1 = act1 ? idx : lc1;
          }
        }
      }
      warp_done = __all_sync(kFullMask, done0 && done1);
    }
  }
}

// Block -> (view, tile) of a batched blend launch: blocks run over the views' tiles in the order
// of tile_base (the host lays the views out heaviest tiles first).
__device__ __forceinline__ TileJob batch_tile_job(const BatchRenderParams& p, uint32_t block) {
  int v = p.tile_order[0];
#pragma unroll 1
  for (int k = 1; k < p.V; ++k) {
    const int w = p.tile_order[k];
    if (p.views[w].tile_base <= block) v = w;
  }
  const BatchView& bv = p.views[v];
  const uint32_t local = block - bv.tile_base;
  TileJob job;
  job.tile_y = (int)(local / (uint32_t)bv.gx);
  job.tile_x = (int)(local - (uint32_t)job.tile_y * (uint32_t)bv.gx);
  job.W = bv.W;
  job.H = bv.H;
  job.range = checked_range(p.ranges, block, p.capacity);
  job.bg = p.backgrounds + 3 * v;
  job.out_color = bv.out_color;
  job.final_T = p.final_T + bv.pixel_base;
  job.n_contrib = p.n_contrib + bv.pixel_base;
  job.dL_dpix = bv.dL_dpix;
  job.wrap_w = p.seam_wrap ? (float)bv.W : 0.f;
  return job;
}

}  // namespace omnigs
