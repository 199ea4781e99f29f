// C-ABI entry points of the batched multi-view path (include/omnigs_b200.h, "batched views"):
// validation, state carving and the launch sequence.  Every stage is one launch for all views:
//   forward:  batched preprocess -> segmented depth sort (one segment per view) -> duplicate over
//             all views (global tile ids) -> tile sort -> ranges -> blend of every view's tiles;
//   backward: blend backward of every view's tiles -> batched backward preprocess.
// The views' tiles are numbered smallest image first: a small equirect image packs more
// Gaussians into each tile, so its blocks are the longest and start first.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>

#include "../../include/omnigs_b200.h"
#include "capi_internal.h"
#include "kernels.h"

namespace omnigs {
namespace {

// Tile and pixel numbering of a batch, computed on the host from the view sizes.
struct BatchPlan {
  int V = 0;
  int64_t pixels = 0, tiles = 0;
  int64_t pixel_base[kMaxBatchViews] = {};
  int64_t tile_base[kMaxBatchViews] = {};
  int64_t view_tiles[kMaxBatchViews] = {};
  uint8_t tile_order[kMaxBatchViews] = {};
  int P = 0;
};

// The tile sort of a batch.  Each view's instances leave the duplicate pass contiguous (view after
// view), so the sort can run per view on view-local tile ids, which need fewer digits than the
// batch's global ids when the views together hold more than 2^k tiles and the largest alone fewer.
// Per view, each segment has its own digit histograms (counted by the duplicate pass's emission)
// and its own look-back chain.
struct BatchTileSort {
  TileDigits digits;
  bool per_view;
};

BatchTileSort batch_tile_sort(const BatchPlan& plan) {
  const TileDigits global = TileDigits::from_tiles((uint32_t)plan.tiles);
  int64_t max_view_tiles = 1;
  for (int v = 0; v < plan.V; ++v) max_view_tiles = std::max(max_view_tiles, plan.view_tiles[v]);
  const TileDigits local = TileDigits::from_tiles((uint32_t)max_view_tiles);
  const bool per_view = plan.V > 1 && local.passes < global.passes;
  return {per_view ? local : global, per_view};
}

int make_plan(int P, int V, const int* W, const int* H, BatchPlan& plan) {
  if (P < 0) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P must be >= 0");
  if (V < 1 || V > kMaxBatchViews)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "the number of views must be in [1, OMNIGS_MAX_BATCH_VIEWS]");
  if (W == nullptr || H == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "view sizes are required");
  if ((int64_t)P * V > (int64_t(1) << 31))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P * V must be at most 2^31 (records are indexed by 32 bits)");
  plan.V = V;
  plan.P = P;
  int64_t order[kMaxBatchViews];
  for (int v = 0; v < V; ++v) {
    if (W[v] <= 0 || H[v] <= 0 || W[v] > 65536 || H[v] > 65536 || (int64_t)W[v] * H[v] > (int64_t(1) << 28))
      return fail(OMNIGS_ERR_INVALID_ARGUMENT, "every view must be positive and at most 2^28 pixels");
    plan.pixel_base[v] = plan.pixels;
    plan.pixels += (int64_t)W[v] * H[v];
    order[v] = v;
  }
  // smallest images first (stable by view index)
  std::stable_sort(order, order + V, [&](int64_t a, int64_t b) {
    return (int64_t)W[a] * H[a] < (int64_t)W[b] * H[b];
  });
  for (int k = 0; k < V; ++k) {
    const int v = (int)order[k];
    plan.tile_order[k] = (uint8_t)v;
    plan.tile_base[v] = plan.tiles;
    plan.view_tiles[v] = (int64_t)tiles_x(W[v]) * tiles_y(H[v]);
    plan.tiles += plan.view_tiles[v];
  }
  if (plan.pixels > 0xffffffffll)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a batch holds at most 2^32 - 1 pixels");
  if (plan.tiles >= (int64_t(1) << (kTilePasses * kRadixBits)))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a batch holds at most 2^24 - 1 tiles");
  return OMNIGS_OK;
}

int plan_from_args(const OmnigsBatchArgs* a, BatchPlan& plan) {
  if (a == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "args is NULL");
  if (a->V < 1 || a->V > kMaxBatchViews || a->views == nullptr)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "the number of views must be in [1, OMNIGS_MAX_BATCH_VIEWS]");
  int W[kMaxBatchViews], H[kMaxBatchViews];
  for (int v = 0; v < a->V; ++v) {
    W[v] = a->views[v].W;
    H[v] = a->views[v].H;
  }
  return make_plan(a->P, a->V, W, H, plan);
}

int validate_batch(const OmnigsBatchArgs* a, BatchPlan& plan) {
  if (int rc = plan_from_args(a, plan)) return rc;
  if (a->sh_dtype != OMNIGS_SH_FP32 && a->sh_dtype != OMNIGS_SH_BF16)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "sh_dtype must be OMNIGS_SH_FP32 or OMNIGS_SH_BF16");
  if (a->fp64_poles != 0 && a->fp64_poles != 1) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "fp64_poles must be 0 or 1");
  if (a->seam_wrap != 0 && a->seam_wrap != 1) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "seam_wrap must be 0 or 1");
  if (a->shs != nullptr && a->M > 16)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "batched views support at most 16 SH coefficients per Gaussian");
  if (int rc = validate_common(a->P, a->D, a->M, a->views[0].W, a->views[0].H, a->shs, a->colors_precomp, a->scales,
                               a->rotations, a->cov3D_precomp, a->means3D, a->viewmatrices, a->campos))
    return rc;
  if (a->backgrounds == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "backgrounds are required");
  if (a->P > 0 && a->opacities == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "opacities are required");
  return OMNIGS_OK;
}

BatchLayout batch_layout(int P, const BatchPlan& plan) { return BatchLayout::make(P, plan.V, plan.pixels, plan.tiles); }

// Kernel parameters common to the batched preprocess passes.
BatchParams batch_params(const OmnigsBatchArgs* a, const BatchPlan& plan, void* state, const BatchLayout& L) {
  BatchParams p{};
  p.P = a->P;
  p.V = a->V;
  p.D = a->D;
  p.M = a->shs != nullptr ? a->M : 0;
  p.sh_bf16 = a->sh_dtype == OMNIGS_SH_BF16;
  p.seam_wrap = a->seam_wrap;
  p.total_tiles = (uint32_t)plan.tiles;
  p.means3D = a->means3D;
  p.scales = a->scales;
  p.rotations = a->rotations;
  p.opacities = a->opacities;
  p.shs = a->shs;
  p.colors_precomp = a->colors_precomp;
  p.cov3D_precomp = a->cov3D_precomp;
  p.scale_modifier = a->scale_modifier;
  p.viewmatrices = a->viewmatrices;
  p.campos = a->campos;
  p.backgrounds = a->backgrounds;
  p.radii = at<int>(state, L.radii);
  p.splat = at<float4>(state, L.splat);
  p.color = at<float4>(state, L.color);
  p.depth = at<float>(state, L.depth);
  p.grad_acc = at<float4>(state, L.grad_acc);
  p.hdr = at<GeomHeader>(state, L.header);
  p.view_rendered = at<unsigned long long>(state, L.view_rendered);
  for (int v = 0; v < a->V; ++v) {
    BatchView& bv = p.views[v];
    bv.W = a->views[v].W;
    bv.H = a->views[v].H;
    bv.gx = tiles_x(bv.W);
    bv.gy = tiles_y(bv.H);
    bv.tile_base = (uint32_t)plan.tile_base[v];
    bv.pixel_base = (uint32_t)plan.pixel_base[v];
    bv.out_color = a->views[v].out_color;
    bv.dL_dpix = a->views[v].dL_dout_color;
  }
  return p;
}

BatchRenderParams render_params(const BatchParams& p, const BatchPlan& plan, void* state, const BatchLayout& L,
                                const uint32_t* point_list, int64_t capacity) {
  BatchRenderParams r{};
  r.P = p.P;
  r.V = p.V;
  r.ranges = at<uint2>(state, L.ranges);
  r.point_list = point_list;
  r.capacity = capacity;
  r.splat = p.splat;
  r.color = p.color;
  r.backgrounds = p.backgrounds;
  r.final_T = at<float>(state, L.final_T);
  r.n_contrib = at<uint32_t>(state, L.n_contrib);
  r.grad_acc = reinterpret_cast<float*>(p.grad_acc);
  r.total_tiles = (uint32_t)plan.tiles;
  r.seam_wrap = p.seam_wrap;
  for (int v = 0; v < p.V; ++v) {
    r.views[v] = p.views[v];
    r.tile_order[v] = plan.tile_order[v];
  }
  return r;
}

int check_state(const BatchLayout& L, void* state, size_t state_bytes) {
  if (state == nullptr || state_bytes < L.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "batch state smaller than omnigs_batch_state_bytes()");
  return check_aligned(state);
}

}  // namespace
}  // namespace omnigs

using namespace omnigs;

extern "C" {

size_t omnigs_batch_state_bytes(int P, int V, const int* W, const int* H) {
  BatchPlan plan;
  if (make_plan(P, V, W, H, plan)) return 0;
  return batch_layout(P, plan).total;
}

int omnigs_batch_render(const OmnigsBatchArgs* a, void* state, size_t state_bytes, void* binning,
                        size_t binning_bytes, omnigs_stream_t stream) {
  g_last_error.clear();
  BatchPlan plan;
  if (int rc = validate_batch(a, plan)) return rc;
  for (int v = 0; v < a->V; ++v)
    if (a->views[v].out_color == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "every view needs out_color");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->P == 0) {
    for (int v = 0; v < a->V; ++v)
      if (cudaMemsetAsync(a->views[v].out_color, 0, sizeof(float) * 3 * a->views[v].W * a->views[v].H, s) !=
          cudaSuccess)
        return check_launch("memset out_color");
    return OMNIGS_OK;
  }
  const BatchLayout L = batch_layout(a->P, plan);
  if (int rc = check_state(L, state, state_bytes)) return rc;
  int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (binning == nullptr || capacity < 0)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer smaller than omnigs_lonlat_binning_bytes(0)");
  if (int rc = check_aligned(binning)) return rc;
  const BinningLayout BL = BinningLayout::make(capacity);
  if (capacity > kMaxInstances) capacity = kMaxInstances;
  const BatchParams bp = batch_params(a, plan, state, L);
  GeomHeader* hdr = bp.hdr;
  uint32_t* thist = at<uint32_t>(binning, BL.hist);
  uint32_t* dhist = at<uint32_t>(state, L.depth_hist);
  const int64_t records = (int64_t)a->P * a->V;
  const int64_t inst_tiles = sort_tiles(BL.capacity);

  staged(OMNIGS_STAGE_OTHER, 1, s, [&] { launch_begin_render(hdr, s); });
  if (cudaMemsetAsync(at<unsigned char>(state, L.dup_scan), 0, L.zero_end - L.dup_scan, s) != cudaSuccess ||
      cudaMemsetAsync(thist, 0, sizeof(uint32_t) * kMaxSortPasses * kRadix, s) != cudaSuccess ||
      cudaMemsetAsync(at<uint2>(state, L.ranges), 0, sizeof(uint2) * plan.tiles, s) != cudaSuccess)
    return check_launch("memset batch binning state");

  // 1. depth sort of every view's Gaussians: one segment per view, (depth bits, index) order
  const uint32_t* depth_keys = reinterpret_cast<const uint32_t*>(bp.depth);
  uint32_t* dkeys[2] = {at<uint32_t>(state, L.dkeys0), at<uint32_t>(state, L.dkeys1)};
  uint32_t* dvals[2] = {at<uint32_t>(state, L.dvals0), at<uint32_t>(state, L.dvals1)};
  HistParams hd{};
  hd.keys = depth_keys;
  hd.n_host = (uint32_t)records;
  hd.passes = kDepthPasses;
  for (int q = 0; q < kDepthPasses; ++q) {
    hd.shift[q] = kRadixBits * q;
    hd.mask[q] = kRadix - 1;
  }
  hd.hist = dhist;
  hd.seg_len = (uint32_t)a->P;
  hd.num_segs = (uint32_t)a->V;
  staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_histogram(hd, records, s); });
  const int64_t depth_tiles = sort_tiles(a->P) * a->V;
  for (int q = 0; q < kDepthPasses; ++q) {
    OnesweepParams op{};
    op.keys_in = q == 0 ? depth_keys : dkeys[(q + 1) & 1];
    op.vals_in = q == 0 ? nullptr : dvals[(q + 1) & 1];
    op.keys_out = dkeys[q & 1];
    op.vals_out = dvals[q & 1];
    op.shift = kRadixBits * q;
    op.mask = kRadix - 1;
    op.n_host = (uint32_t)records;
    op.hist = dhist + q * kRadix;
    op.lookback = at<uint32_t>(state, L.depth_lookback) + (size_t)q * depth_tiles * kRadix;
    op.tile_counter = &hdr->sort_tile_counter[q];
    op.hdr = hdr;
    op.seg_len = (uint32_t)a->P;
    op.num_segs = (uint32_t)a->V;
    op.hist_seg_stride = kDepthPasses * kRadix;
    staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_onesweep(op, records, s); });
  }
  const uint32_t* order = dvals[(kDepthPasses - 1) & 1];

  // 2. duplicate every view's instances in that order, keyed by global tile id
  uint32_t* tkeys[2] = {at<uint32_t>(binning, BL.tkeys0), at<uint32_t>(binning, BL.tkeys1)};
  uint32_t* tvals[2] = {at<uint32_t>(binning, BL.tvals0), at<uint32_t>(binning, BL.tvals1)};
  DuplicateParams d{};
  d.P = a->P;
  d.V = a->V;
  d.radii = bp.radii;
  d.splat = bp.splat;
  d.order = order;
  d.tkeys = tkeys[0];
  d.tvals = tvals[0];
  d.scan_state = at<unsigned long long>(state, L.dup_scan);
  d.incl = dkeys[0];  // free once the last depth pass has read it (the sorted keys are in dkeys[1])
  // the depth sort's other free buffers: its sorted keys and its first value buffer
  static_assert(((kDepthPasses - 1) & 1) == 1, "the depth order is in dvals[1]");
  d.rect_row = dvals[0];
  d.rect_cw = dkeys[1];
  d.emit_first = at<uint32_t>(binning, BL.emit_first);
  d.emit_last = at<uint32_t>(binning, BL.emit_last);
  d.capacity = capacity;
  d.hdr = hdr;
  d.seam_wrap = a->seam_wrap;
  for (int v = 0; v < a->V; ++v) {
    d.gx[v] = bp.views[v].gx;
    d.gy[v] = bp.views[v].gy;
    d.tile_base[v] = bp.views[v].tile_base;
  }
  // tile sort per view or over the global tile ids (batch_tile_sort)
  const BatchTileSort ts = batch_tile_sort(plan);
  const bool per_view = ts.per_view;
  const TileDigits& tds = ts.digits;
  uint32_t* tile_hist = per_view ? at<uint32_t>(state, L.tile_hist) : thist + kDepthPasses * kRadix;
  const int64_t lb_tiles = inst_tiles + a->V;  // look-back tiles per pass (per view: partial tiles)
  if (cudaMemsetAsync(at<uint32_t>(binning, BL.tile_lookback), 0, sizeof(uint32_t) * tds.passes * lb_tiles * kRadix,
                      s) != cudaSuccess)
    return check_launch("memset tile look-back");
  d.hist = tile_hist;
  d.hist_passes = tds.passes;
  d.hist_per_view = per_view ? 1 : 0;
  d.key_base_out = at<uint32_t>(state, L.view_key_base);
  for (int q = 0; q < tds.passes; ++q) {
    d.hist_shift[q] = tds.shift[q];
    d.hist_mask[q] = tds.mask[q];
  }
  staged(OMNIGS_STAGE_DUPLICATE, 1, s, [&] { launch_duplicate(d, s); });

  // 3. stable tile sort of all instances (per view when per_view; the digit histograms were
  // counted by the duplicate pass)
  for (int q = 0; q < tds.passes; ++q) {
    OnesweepParams op{};
    op.keys_in = tkeys[q & 1];
    op.vals_in = tvals[q & 1];
    op.keys_out = tkeys[(q + 1) & 1];
    op.vals_out = tvals[(q + 1) & 1];
    op.shift = tds.shift[q];
    op.mask = tds.mask[q];
    op.count_hdr = hdr;
    op.capacity = capacity;
    op.hist = tile_hist + q * kRadix;
    op.lookback = at<uint32_t>(binning, BL.tile_lookback) + (size_t)q * lb_tiles * kRadix;
    op.tile_counter = &hdr->sort_tile_counter[kDepthPasses + q];
    op.hdr = hdr;
    if (per_view) {
      op.seg_counts = bp.view_rendered;
      op.num_segs = (uint32_t)a->V;
      op.hist_seg_stride = kTilePasses * kRadix;
      op.add_key_base = q == tds.passes - 1;
    }
    staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_onesweep(op, capacity, s); });
  }
  const int fin = tds.passes & 1;
  if (int rc = check_launch("batch binning")) return rc;

  // 4. tile ranges over all views' tiles
  RangesParams rp{};
  rp.keys = tkeys[fin];
  rp.ranges = at<uint2>(state, L.ranges);
  rp.num_tiles = (uint32_t)plan.tiles;
  rp.capacity = capacity;
  rp.hdr = hdr;
  staged(OMNIGS_STAGE_RANGES, 1, s, [&] { launch_ranges(rp, s); });
  if (int rc = check_launch("batch ranges")) return rc;

  // 5. blend every tile of every view
  const BatchRenderParams r = render_params(bp, plan, state, L, tvals[fin], capacity);
  staged(OMNIGS_STAGE_RENDER_FORWARD, 1, s, [&] { launch_batch_render_forward(r, s); });
  return check_launch("batch render forward");
}

int omnigs_batch_forward(const OmnigsBatchArgs* a, void* state, size_t state_bytes, void* binning,
                         size_t binning_bytes, omnigs_stream_t stream) {
  g_last_error.clear();
  BatchPlan plan;
  if (int rc = validate_batch(a, plan)) return rc;
  if (a->P > 0) {
    const BatchLayout L = batch_layout(a->P, plan);
    if (int rc = check_state(L, state, state_bytes)) return rc;
    if (int rc = check_aligned(binning)) return rc;  // before the preprocess's device work
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(state, 0, L.dup_scan, s) != cudaSuccess) return check_launch("memset batch header");
    const BatchParams bp = batch_params(a, plan, state, L);
    staged(OMNIGS_STAGE_PREPROCESS, 1, s, [&] { launch_batch_preprocess(bp, a->fp64_poles, s); });
    if (int rc = check_launch("batch preprocess")) return rc;
  }
  return omnigs_batch_render(a, state, state_bytes, binning, binning_bytes, stream);
}

int omnigs_batch_backward(const OmnigsBatchArgs* a, const OmnigsBatchGrads* g, void* state, size_t state_bytes,
                          const void* binning, size_t binning_bytes, omnigs_stream_t stream) {
  g_last_error.clear();
  BatchPlan plan;
  if (int rc = validate_batch(a, plan)) return rc;
  if (g == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "grads is NULL");
  if (a->P == 0) return OMNIGS_OK;  // no Gaussians, no gradients (the outputs are empty)
  if (g->dL_dmeans3D == nullptr || g->dL_dopacity == nullptr || g->dL_dscales == nullptr ||
      g->dL_drotations == nullptr || (a->shs != nullptr && a->M > 0 && g->dL_dsh == nullptr))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a required batched gradient output is NULL");
  for (int v = 0; v < a->V; ++v)
    if (a->views[v].dL_dout_color == nullptr)
      return fail(OMNIGS_ERR_INVALID_ARGUMENT, "every view needs dL_dout_color");
  const BatchLayout L = batch_layout(a->P, plan);
  if (int rc = check_state(L, state, state_bytes)) return rc;
  int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (binning == nullptr || capacity < 0)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer smaller than omnigs_lonlat_binning_bytes(0)");
  if (int rc = check_aligned(binning)) return rc;
  const BinningLayout BL = BinningLayout::make(capacity);
  if (capacity > kMaxInstances) capacity = kMaxInstances;
  const int fin = batch_tile_sort(plan).digits.passes & 1;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const BatchParams bp = batch_params(a, plan, state, L);
  const BatchRenderParams r =
      render_params(bp, plan, state, L, at<uint32_t>(binning, fin ? BL.tvals1 : BL.tvals0), capacity);
  staged(OMNIGS_STAGE_RENDER_BACKWARD, 1, s, [&] { launch_batch_render_backward(r, s); });
  if (int rc = check_launch("batch render backward")) return rc;
  BatchGrads bg{};
  bg.dL_dmeans3D = g->dL_dmeans3D;
  bg.dL_dsh = a->shs != nullptr ? g->dL_dsh : nullptr;
  bg.dL_dopacity = g->dL_dopacity;
  bg.dL_dscales = g->dL_dscales;
  bg.dL_drotations = g->dL_drotations;
  bg.dL_dcolors = g->dL_dcolors;
  bg.dL_dcov3D = g->dL_dcov3D;
  bg.grad_accum = g->grad_accum;
  bg.denom = g->denom;
  bg.max_radii = g->max_radii;
  staged(OMNIGS_STAGE_PREPROCESS_BACKWARD, 1, s,
         [&] { launch_batch_preprocess_backward(bp, bg, a->fp64_poles, s); });
  return check_launch("batch preprocess backward");
}

int omnigs_batch_autotune(const OmnigsBatchArgs* a, void* state, size_t state_bytes, void* binning,
                          size_t binning_bytes, int repeats, OmnigsTuneResult* out, omnigs_stream_t stream) {
  g_last_error.clear();
  BatchPlan plan;
  if (int rc = validate_batch(a, plan)) return rc;
  if (out == nullptr || repeats < 1) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "out is NULL or repeats < 1");
  for (int v = 0; v < a->V; ++v)
    if (a->views[v].out_color == nullptr || a->views[v].dL_dout_color == nullptr)
      return fail(OMNIGS_ERR_INVALID_ARGUMENT, "every view needs out_color and dL_dout_color");
  const int cand[3] = {128, 256, 512};
  std::memset(out, 0, sizeof(*out));
  for (int k = 0; k < 3; ++k) out->candidates[k] = cand[k];
  out->forward_batch = g_blend_batch[0].load();
  out->backward_batch = g_blend_batch[1].load();
  if (a->P == 0) return OMNIGS_OK;
  const BatchLayout L = batch_layout(a->P, plan);
  if (int rc = check_state(L, state, state_bytes)) return rc;
  int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (binning == nullptr || capacity < 0)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer smaller than omnigs_lonlat_binning_bytes(0)");
  if (int rc = check_aligned(binning)) return rc;
  const BinningLayout BL = BinningLayout::make(capacity);
  if (capacity > kMaxInstances) capacity = kMaxInstances;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  GeomHeader h;
  if (cudaMemcpyAsync(&h, state, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return check_launch("read batch status");
  if (h.status != 0)
    return fail(OMNIGS_ERR_DEVICE, "the batch state holds no complete forward (status word set); run omnigs_batch_forward first");
  const int fin = batch_tile_sort(plan).digits.passes & 1;
  const BatchParams bp = batch_params(a, plan, state, L);
  const BatchRenderParams r =
      render_params(bp, plan, state, L, at<uint32_t>(binning, fin ? BL.tvals1 : BL.tvals0), capacity);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return check_launch("events");
  const int saved[2] = {g_blend_batch[0].load(), g_blend_batch[1].load()};
  int rc = OMNIGS_OK;
  for (int dir = 0; dir < 2 && rc == OMNIGS_OK; ++dir) {
    float best = 0.f;
    int best_b = saved[dir];
    for (int k = 0; k < 3; ++k) {
      g_blend_batch[dir].store(cand[k]);
      auto launch = [&] {
        if (dir == 0)
          launch_batch_render_forward(r, s);
        else
          launch_batch_render_backward(r, s);
        g_launches.fetch_add(1, std::memory_order_relaxed);
      };
      launch();  // warm-up
      cudaEventRecord(e0, s);
      for (int t = 0; t < repeats; ++t) launch();
      cudaEventRecord(e1, s);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = check_launch("autotune timing");
        break;
      }
      ms /= repeats;
      (dir == 0 ? out->forward_ms : out->backward_ms)[k] = ms;
      if (k == 0 || ms < best) {
        best = ms;
        best_b = cand[k];
      }
    }
    g_blend_batch[dir].store(rc == OMNIGS_OK ? best_b : saved[dir]);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  out->forward_batch = g_blend_batch[0].load();
  out->backward_batch = g_blend_batch[1].load();
  // the timed backward launches summed into the accumulators: clear them for the real backward
  if (cudaMemsetAsync(at<unsigned char>(state, L.grad_acc), 0, sizeof(float) * 12 * (size_t)a->P * a->V, s) !=
      cudaSuccess)
    return check_launch("clear accumulators");
  return check_launch("autotune");
}

int omnigs_batch_read_status(const void* state, int V, int64_t* num_rendered, int64_t* view_rendered,
                             uint32_t* status, omnigs_stream_t stream) {
  g_last_error.clear();
  if (state == nullptr || V < 1 || V > kMaxBatchViews)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad batch status arguments");
  struct {
    GeomHeader h;
    unsigned long long views[32];
  } host;
  static_assert(sizeof(GeomHeader) == kAlign, "the per-view counts follow the header");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(&host, state, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return check_launch("read batch status");
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_launch("synchronize");
  if (num_rendered) *num_rendered = (int64_t)host.h.num_rendered64;
  if (view_rendered)
    for (int v = 0; v < V; ++v) view_rendered[v] = (int64_t)host.views[v];
  if (status) *status = host.h.status;
  return OMNIGS_OK;
}

int omnigs_batch_state_view(const void* state, int P, int V, const int* W, const int* H, OmnigsBatchStateView* out) {
  g_last_error.clear();
  if (state == nullptr || out == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad view arguments");
  BatchPlan plan;
  if (int rc = make_plan(P, V, W, H, plan)) return rc;
  const BatchLayout L = batch_layout(P, plan);
  std::memset(out, 0, sizeof(*out));
  out->radii = at<int>(state, L.radii);
  out->splat = at<float>(state, L.splat);
  out->color = at<float>(state, L.color);
  out->final_T = at<float>(state, L.final_T);
  out->n_contrib = at<uint32_t>(state, L.n_contrib);
  out->ranges = at<uint32_t>(state, L.ranges);
  for (int v = 0; v < V; ++v) {
    out->pixel_base[v] = plan.pixel_base[v];
    out->tile_base[v] = plan.tile_base[v];
  }
  out->tile_passes = batch_tile_sort(plan).digits.passes;
  out->depth = at<float>(state, L.depth);
  return OMNIGS_OK;
}

int omnigs_batch_binning_view(const void* binning, size_t binning_bytes, int P, int V, const int* W, const int* H,
                              OmnigsLonlatBinningView* out) {
  g_last_error.clear();
  if (binning == nullptr || out == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad view arguments");
  BatchPlan plan;
  if (int rc = make_plan(P, V, W, H, plan)) return rc;
  const int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (capacity < 0) return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer too small");
  const BinningLayout BL = BinningLayout::make(capacity);
  const int fin = batch_tile_sort(plan).digits.passes & 1;
  out->tile_ids = at<uint32_t>(binning, fin ? BL.tkeys1 : BL.tkeys0);
  out->point_list = at<uint32_t>(binning, fin ? BL.tvals1 : BL.tvals0);
  return OMNIGS_OK;
}

}  // extern "C"
