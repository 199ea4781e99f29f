// C-ABI entry points (include/omnigs_b200.h): argument validation, buffer carving and kernel
// sequencing for one lonlat rasterization.  Replaces the host orchestration of
// CudaRasterizer::LonlatRasterizer (rasterizer_impl.cu:540-795) without its mid-pass host sync.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/omnigs_b200.h"
#include "capi_internal.h"
#include "kernels.h"

namespace omnigs {

thread_local std::string g_last_error;

int fail(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return OMNIGS_ERR_CUDA;
  }
  return OMNIGS_OK;
}

std::atomic<uint64_t> g_launches{0};
std::atomic<bool> g_timing{false};
std::mutex g_timing_mu;
std::vector<TimedLaunch> g_timed;
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t take_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

__global__ void begin_render_kernel(GeomHeader* hdr) {
  atomicAnd(&hdr->status, ~(kStatusCapacity | kStatusInconsistent));
  const unsigned long long total = hdr->num_rendered64;
  if (total > (unsigned long long)kMaxInstances) atomicOr(&hdr->status, kStatusOverflow);
  hdr->num_rendered = (uint32_t)(total > 0xffffffffull ? 0xffffffffull : total);
  hdr->dup_tile_counter = 0;
  for (int i = 0; i < kMaxSortPasses; ++i) hdr->sort_tile_counter[i] = 0;
}

void launch_begin_render(GeomHeader* hdr, cudaStream_t s) { begin_render_kernel<<<1, 1, 0, s>>>(hdr); }

int check_aligned(const void* a, const void* b, const void* c) {
  for (const void* q : {a, b, c})
    if ((reinterpret_cast<uintptr_t>(q) & 15) != 0)
      return fail(OMNIGS_ERR_INVALID_ARGUMENT, "workspace buffers must be 16-byte aligned");
  return OMNIGS_OK;
}

int validate_common(int P, int D, int M, int W, int H, const void* shs, const float* colors,
                    const float* scales, const float* rotations, const float* cov3D,
                    const float* means3D, const float* viewmatrix, const float* campos) {
  if (P < 0) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P must be >= 0");
  if (W <= 0 || H <= 0 || W > 65536 || H > 65536 || (int64_t)W * H > (int64_t(1) << 28))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "image size must be positive and at most 2^28 pixels");
  if (P == 0) return OMNIGS_OK;
  if (D < 0 || D > 3) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "SH degree must be in [0, 3]");
  if ((shs == nullptr) == (colors == nullptr))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "Please provide excatly one of either SHs or precomputed colors!");
  if (shs != nullptr && M < (D + 1) * (D + 1))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "sh has fewer coefficients per Gaussian than the SH degree needs");
  const bool have_sr = scales != nullptr || rotations != nullptr;
  if ((have_sr && cov3D != nullptr) || (!have_sr && cov3D == nullptr) ||
      (have_sr && (scales == nullptr || rotations == nullptr)))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT,
                "Please provide exactly one of either scale/rotation pair or precomputed 3D covariance!");
  if (means3D == nullptr || viewmatrix == nullptr || (shs != nullptr && campos == nullptr))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "means3D, viewmatrix and campos are required");
  return OMNIGS_OK;
}

namespace {

// Buffer (0 or 1) that holds the sorted tile ids / point list after the tile passes.
int tile_final(int W, int H) { return TileDigits::make(W, H).passes & 1; }

int validate_forward(const OmnigsLonlatForwardArgs* a) {
  if (a == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "args is NULL");
  const int rc = validate_common(a->P, a->D, a->M, a->W, a->H, a->shs, a->colors_precomp, a->scales,
                                 a->rotations, a->cov3D_precomp, a->means3D, a->viewmatrix, a->campos);
  if (rc) return rc;
  if (a->out_color == nullptr || a->background == nullptr)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "out_color and background are required");
  if (a->P > 0 && (a->radii == nullptr || a->opacities == nullptr))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "radii and opacities are required");
  if (a->flags & ~OMNIGS_FLAG_RECOMPUTE_T) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "unknown flags");
  return OMNIGS_OK;
}

// Per-pixel state is stored unless the caller asked for transmittance checkpointing.
bool stores_state(int flags) { return (flags & OMNIGS_FLAG_RECOMPUTE_T) == 0; }

__global__ void mark_visible_kernel(int P, const float* means3D, const float* vm, int camera_type,
                                    uint8_t* present) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= P) return;
  if (camera_type == OMNIGS_CAMERA_LONLAT) {
    present[idx] = 1;
    return;
  }
  const float x = means3D[3 * idx], y = means3D[3 * idx + 1], z = means3D[3 * idx + 2];
  const float pz = vm[2] * x + vm[6] * y + vm[10] * z + vm[14];
  present[idx] = (pz <= 0.2f) ? 0 : 1;
}

}  // namespace

void set_last_error(const char* msg) { g_last_error = msg; }

std::atomic<int> g_blend_batch[2] = {{kDefaultBatch}, {kDefaultBwdBatch}};
int blend_batch_size(bool backward) { return g_blend_batch[backward ? 1 : 0].load(std::memory_order_relaxed); }

void launch_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                         bool* present, cudaStream_t s) {
  if (P <= 0) return;
  mark_visible_kernel<<<(P + 255) / 256, 256, 0, s>>>(P, means3D, viewmatrix, camera_type,
                                                        reinterpret_cast<uint8_t*>(present));
}

}  // namespace omnigs

using namespace omnigs;

extern "C" {

const char* omnigs_version(void) { return "omnigs_b200 0.1.0 (sm_100a)"; }

const char* omnigs_last_error(void) { return g_last_error.c_str(); }

size_t omnigs_lonlat_geom_bytes(int P) { return GeomLayout::make(P < 0 ? 0 : P).total; }

size_t omnigs_lonlat_image_bytes(int W, int H) {
  if (W <= 0 || H <= 0) return 0;
  return ImageLayout::make(W, H).total;
}

size_t omnigs_lonlat_image_bytes_flags(int W, int H, int flags) {
  if (W <= 0 || H <= 0) return 0;
  return ImageLayout::make(W, H, stores_state(flags)).total;
}

size_t omnigs_lonlat_binning_bytes(int64_t capacity) {
  return BinningLayout::make(capacity < 0 ? 0 : capacity).total;
}

int64_t omnigs_lonlat_binning_capacity(size_t binning_bytes) {
  return BinningLayout::capacity_for(binning_bytes);
}

int omnigs_lonlat_preprocess(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes,
                             omnigs_stream_t stream) {
  g_last_error.clear();
  if (int rc = validate_forward(a)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const GeomLayout L = GeomLayout::make(a->P);
  if (geom == nullptr || geom_bytes < L.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "geometry buffer smaller than omnigs_lonlat_geom_bytes(P)");
  if (int rc = check_aligned(geom)) return rc;
  if (cudaMemsetAsync(geom, 0, sizeof(GeomHeader), s) != cudaSuccess) return check_launch("memset geometry header");
  if (a->P == 0) return OMNIGS_OK;
  PreprocessParams p{};
  p.P = a->P;
  p.D = a->D;
  p.M = a->M;
  p.W = a->W;
  p.H = a->H;
  p.gx = tiles_x(a->W);
  p.gy = tiles_y(a->H);
  p.means3D = a->means3D;
  p.scales = a->scales;
  p.rotations = a->rotations;
  p.opacities = a->opacities;
  p.shs = a->shs;
  p.colors_precomp = a->colors_precomp;
  p.cov3D_precomp = a->cov3D_precomp;
  p.scale_modifier = a->scale_modifier;
  p.viewmatrix = a->viewmatrix;
  p.campos = a->campos;
  p.radii = a->radii;
  p.splat = at<float4>(geom, L.splat);
  p.color = at<float4>(geom, L.color);
  p.depth = at<float>(geom, L.depth);
  p.tiles_touched = at<uint32_t>(geom, L.tiles_touched);
  p.grad_acc = at<float4>(geom, L.grad_acc);
  p.hdr = at<GeomHeader>(geom, L.header);
  staged(OMNIGS_STAGE_PREPROCESS, 1, s, [&] { launch_preprocess(p, s); });
  return check_launch("preprocess");
}

namespace {

// Pinned host copy of the geometry header and the event recorded after the copy, one per host
// thread and device, for omnigs_lonlat_forward_early_status.  Created on first use and kept for
// the life of the process.
struct EarlyStatus {
  GeomHeader* host = nullptr;
  cudaEvent_t copied = nullptr;
};

EarlyStatus* early_status_slot() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  thread_local std::vector<EarlyStatus> slots;
  if ((int)slots.size() <= dev) slots.resize(dev + 1);
  EarlyStatus& e = slots[dev];
  if (e.host == nullptr) {
    if (cudaHostAlloc(reinterpret_cast<void**>(&e.host), sizeof(GeomHeader), cudaHostAllocDefault) != cudaSuccess) {
      e.host = nullptr;
      return nullptr;
    }
    if (cudaEventCreateWithFlags(&e.copied, cudaEventDisableTiming) != cudaSuccess) {
      cudaFreeHost(e.host);
      e.host = nullptr;
      return nullptr;
    }
  }
  return &e;
}

// A forward cut short after the duplicate pass, whose scan tile 0 is taken by no block and whose
// look-back waits give up after max_spins polls (omnigs_debug_lookback_timeout).
struct LookbackProbe {
  int max_spins;
};

// Binning + forward blend.  With `early`, the header (instance count, status word; final once the
// binning kernels have run) is copied to early->host and early->copied recorded between the binning
// and the blend.  With `probe`, the pass stops after the duplicate kernel (see LookbackProbe).
int render_impl(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes, void* binning,
                size_t binning_bytes, void* image, size_t image_bytes, omnigs_stream_t stream,
                EarlyStatus* early, const LookbackProbe* probe = nullptr) {
  if (int rc = validate_forward(a)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t HW = (int64_t)a->W * a->H;
  if (a->P == 0) {
    // The reference returns its zero-initialised image when there are no Gaussians
    // (src/rasterize_points.cu:84, 97).
    if (cudaMemsetAsync(a->out_color, 0, sizeof(float) * 3 * HW, s) != cudaSuccess)
      return check_launch("memset out_color");
    return OMNIGS_OK;
  }
  const GeomLayout GL = GeomLayout::make(a->P);
  const ImageLayout IL = ImageLayout::make(a->W, a->H, stores_state(a->flags));
  if (geom == nullptr || geom_bytes < GL.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "geometry buffer smaller than omnigs_lonlat_geom_bytes(P)");
  if (image == nullptr || image_bytes < IL.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "image buffer smaller than omnigs_lonlat_image_bytes_flags(W, H, flags)");
  int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (binning == nullptr || capacity < 0)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer smaller than omnigs_lonlat_binning_bytes(0)");
  if (int rc = check_aligned(geom, image, binning)) return rc;
  const BinningLayout BL = BinningLayout::make(capacity);
  if (capacity > kMaxInstances) capacity = kMaxInstances;
  const int gx = tiles_x(a->W), gy = tiles_y(a->H);
  const TileDigits td = TileDigits::make(a->W, a->H);
  GeomHeader* hdr = at<GeomHeader>(geom, GL.header);
  uint32_t* hist = at<uint32_t>(binning, BL.hist);
  uint2* ranges = at<uint2>(image, IL.ranges);
  const int64_t depth_tiles = sort_tiles(a->P);
  const int64_t inst_tiles = sort_tiles(BL.capacity);

  staged(OMNIGS_STAGE_OTHER, 1, s, [&] { launch_begin_render(hdr, s); });
  if (cudaMemsetAsync(at<unsigned char>(geom, GL.dup_scan), 0, GL.zero_end - GL.dup_scan, s) != cudaSuccess ||
      cudaMemsetAsync(hist, 0, sizeof(uint32_t) * kMaxSortPasses * kRadix, s) != cudaSuccess ||
      cudaMemsetAsync(at<uint32_t>(binning, BL.tile_lookback), 0,
                      sizeof(uint32_t) * td.passes * inst_tiles * kRadix, s) != cudaSuccess ||
      cudaMemsetAsync(ranges, 0, sizeof(uint2) * (size_t)gx * gy, s) != cudaSuccess)
    return check_launch("memset binning state");

  // 1. depth sort of the Gaussians: (depth bits, index) order
  const uint32_t* depth_keys = at<uint32_t>(geom, GL.depth);
  uint32_t* dkeys[2] = {at<uint32_t>(geom, GL.dkeys0), at<uint32_t>(geom, GL.dkeys1)};
  uint32_t* dvals[2] = {at<uint32_t>(geom, GL.dvals0), at<uint32_t>(geom, GL.dvals1)};
  HistParams hd{};
  hd.keys = depth_keys;
  hd.n_host = (uint32_t)a->P;
  hd.passes = kDepthPasses;
  for (int q = 0; q < kDepthPasses; ++q) {
    hd.shift[q] = kRadixBits * q;
    hd.mask[q] = kRadix - 1;
  }
  hd.hist = hist;
  staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_histogram(hd, a->P, s); });
  for (int q = 0; q < kDepthPasses; ++q) {
    OnesweepParams op{};
    op.keys_in = q == 0 ? depth_keys : dkeys[(q + 1) & 1];
    op.vals_in = q == 0 ? nullptr : dvals[(q + 1) & 1];
    op.keys_out = dkeys[q & 1];
    op.vals_out = dvals[q & 1];
    op.shift = kRadixBits * q;
    op.mask = kRadix - 1;
    op.n_host = (uint32_t)a->P;
    op.hist = hist + q * kRadix;
    op.lookback = at<uint32_t>(geom, GL.depth_lookback) + (size_t)q * depth_tiles * kRadix;
    op.tile_counter = &hdr->sort_tile_counter[q];
    op.hdr = hdr;
    staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_onesweep(op, a->P, s); });
  }
  const uint32_t* order = dvals[(kDepthPasses - 1) & 1];

  // 2. duplicate in that order (fused scan of the tile counts)
  uint32_t* tkeys[2] = {at<uint32_t>(binning, BL.tkeys0), at<uint32_t>(binning, BL.tkeys1)};
  uint32_t* tvals[2] = {at<uint32_t>(binning, BL.tvals0), at<uint32_t>(binning, BL.tvals1)};
  DuplicateParams d{};
  d.P = a->P;
  d.V = 1;
  d.gx[0] = gx;
  d.gy[0] = gy;
  d.tile_base[0] = 0;
  d.radii = a->radii;
  d.splat = at<float4>(geom, GL.splat);
  d.order = order;
  d.tkeys = tkeys[0];
  d.tvals = tvals[0];
  d.scan_state = at<unsigned long long>(geom, GL.dup_scan);
  d.incl = dkeys[0];  // free once the last depth pass has read it (the sorted keys are in dkeys[1])
  // the depth sort's other free buffers: its sorted keys and its first value buffer
  static_assert(((kDepthPasses - 1) & 1) == 1, "the depth order is in dvals[1]");
  d.rect_row = dvals[0];
  d.rect_cw = dkeys[1];
  d.emit_first = at<uint32_t>(binning, BL.emit_first);
  d.emit_last = at<uint32_t>(binning, BL.emit_last);
  d.capacity = capacity;
  d.hdr = hdr;
  d.hist = hist + kDepthPasses * kRadix;
  d.hist_passes = td.passes;
  for (int q = 0; q < td.passes; ++q) {
    d.hist_shift[q] = td.shift[q];
    d.hist_mask[q] = td.mask[q];
  }
  if (probe != nullptr) {
    d.max_spins = probe->max_spins;
    d.skip_tiles = 1;
  }
  staged(OMNIGS_STAGE_DUPLICATE, 1, s, [&] { launch_duplicate(d, s); });
  if (probe != nullptr) return check_launch("duplicate (look-back probe)");

  // 3. stable tile sort of the instances
  // (its digit histograms were counted by the duplicate pass)
  for (int q = 0; q < td.passes; ++q) {
    OnesweepParams op{};
    op.keys_in = tkeys[q & 1];
    op.vals_in = tvals[q & 1];
    op.keys_out = tkeys[(q + 1) & 1];
    op.vals_out = tvals[(q + 1) & 1];
    op.shift = td.shift[q];
    op.mask = td.mask[q];
    op.count_hdr = hdr;
    op.capacity = capacity;
    op.hist = hist + (kDepthPasses + q) * kRadix;
    op.lookback = at<uint32_t>(binning, BL.tile_lookback) + (size_t)q * inst_tiles * kRadix;
    op.tile_counter = &hdr->sort_tile_counter[kDepthPasses + q];
    op.hdr = hdr;
    staged(OMNIGS_STAGE_SORT, 1, s, [&] { launch_onesweep(op, capacity, s); });
  }
  const int fin = td.passes & 1;
  if (int rc = check_launch("binning")) return rc;

  // 4. tile ranges
  RangesParams rp{};
  rp.keys = tkeys[fin];
  rp.ranges = ranges;
  rp.num_tiles = (uint32_t)gx * (uint32_t)gy;
  rp.capacity = capacity;
  rp.hdr = hdr;
  staged(OMNIGS_STAGE_RANGES, 1, s, [&] { launch_ranges(rp, s); });
  if (int rc = check_launch("ranges")) return rc;

  RenderParams r{};
  r.P = a->P;
  r.W = a->W;
  r.H = a->H;
  r.gx = gx;
  r.gy = gy;
  r.ranges = ranges;
  r.point_list = tvals[fin];
  r.capacity = capacity;
  r.splat = at<float4>(geom, GL.splat);
  r.color = at<float4>(geom, GL.color);
  r.bg = a->background;
  r.out_color = a->out_color;
  r.final_T = IL.store_state ? at<float>(image, IL.final_T) : nullptr;
  r.n_contrib = IL.store_state ? at<uint32_t>(image, IL.n_contrib) : nullptr;
  if (early != nullptr) {
    if (cudaMemcpyAsync(early->host, hdr, sizeof(GeomHeader), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaEventRecord(early->copied, s) != cudaSuccess)
      return check_launch("copy status");
  }
  staged(OMNIGS_STAGE_RENDER_FORWARD, 1, s, [&] { launch_render_forward(r, s); });
  return check_launch("render forward");
}

}  // namespace

int omnigs_lonlat_render(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes,
                         void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                         omnigs_stream_t stream) {
  g_last_error.clear();
  return render_impl(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream, nullptr);
}

int omnigs_lonlat_forward(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes,
                          void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                          omnigs_stream_t stream) {
  if (int rc = check_aligned(geom, binning, image)) return rc;  // before the preprocess's device work
  if (int rc = omnigs_lonlat_preprocess(a, geom, geom_bytes, stream)) return rc;
  return omnigs_lonlat_render(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream);
}

int omnigs_lonlat_forward_early_status(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes,
                                       void* binning, size_t binning_bytes, void* image, size_t image_bytes,
                                       int* num_rendered, uint32_t* status, omnigs_stream_t stream) {
  if (num_rendered == nullptr || status == nullptr)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "num_rendered and status must not be NULL");
  if (int rc = check_aligned(geom, binning, image)) return rc;  // before the preprocess's device work
  if (int rc = omnigs_lonlat_preprocess(a, geom, geom_bytes, stream)) return rc;
  g_last_error.clear();
  if (a->P == 0) {
    *num_rendered = 0;
    *status = 0;
    return render_impl(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream, nullptr);
  }
  EarlyStatus* e = early_status_slot();
  if (e == nullptr) return fail(OMNIGS_ERR_CUDA, "could not create the pinned status slot");
  if (int rc = render_impl(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream, e)) return rc;
  if (cudaEventSynchronize(e->copied) != cudaSuccess) return check_launch("wait for the binning status");
  const unsigned long long n = e->host->num_rendered64;
  *num_rendered = (int)(n > 0x7fffffffull ? 0x7fffffff : n);
  *status = e->host->status;
  return OMNIGS_OK;
}

int omnigs_debug_lookback_timeout(const OmnigsLonlatForwardArgs* a, void* geom, size_t geom_bytes, void* binning,
                                  size_t binning_bytes, void* image, size_t image_bytes, int max_spins,
                                  uint32_t* status, omnigs_stream_t stream) {
  g_last_error.clear();
  if (a == nullptr || status == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (max_spins <= 0) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "max_spins must be positive");
  if (a->P <= kScanTile)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "the look-back probe needs more than one scan tile of Gaussians");
  if (int rc = omnigs_lonlat_preprocess(a, geom, geom_bytes, stream)) return rc;
  const LookbackProbe probe{max_spins};
  if (int rc = render_impl(a, geom, geom_bytes, binning, binning_bytes, image, image_bytes, stream, nullptr, &probe))
    return rc;
  int n = 0;
  if (int rc = omnigs_lonlat_read_status(geom, &n, status, stream)) return rc;
  if (*status & ~OMNIGS_STATUS_CAPACITY) {
    const std::string msg = "device status " + std::to_string(*status) +
                            (*status & OMNIGS_STATUS_LOOKBACK ? ": a bounded look-back wait gave up" : "");
    return fail(OMNIGS_ERR_DEVICE, msg.c_str());
  }
  return OMNIGS_OK;
}

int omnigs_lonlat_read_status(const void* geom, int* num_rendered, uint32_t* status,
                              omnigs_stream_t stream) {
  g_last_error.clear();
  if (geom == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "geom is NULL");
  GeomHeader h;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(&h, geom, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return check_launch("read status");
  if (cudaStreamSynchronize(s) != cudaSuccess) return check_launch("synchronize");
  if (num_rendered) *num_rendered = (int)(h.num_rendered64 > 0x7fffffffull ? 0x7fffffff : h.num_rendered64);
  if (status) *status = h.status;
  return OMNIGS_OK;
}

int omnigs_lonlat_backward(const OmnigsLonlatBackwardArgs* a, void* geom, size_t geom_bytes,
                           const void* binning, size_t binning_bytes, const void* image,
                           size_t image_bytes, omnigs_stream_t stream) {
  g_last_error.clear();
  if (a == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "args is NULL");
  if (int rc = validate_common(a->P, a->D, a->M, a->W, a->H, a->shs, a->colors_precomp, a->scales,
                               a->rotations, a->cov3D_precomp, a->means3D, a->viewmatrix, a->campos))
    return rc;
  if (a->flags & ~OMNIGS_FLAG_RECOMPUTE_T) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "unknown flags");
  if (a->P == 0) return OMNIGS_OK;
  if (a->radii == nullptr || a->dL_dout_color == nullptr || a->background == nullptr ||
      a->dL_dmeans2D == nullptr || a->dL_dcolors == nullptr || a->dL_dopacity == nullptr ||
      a->dL_dmeans3D == nullptr || a->dL_dcov3D == nullptr || a->dL_dscales == nullptr ||
      a->dL_drotations == nullptr || (a->M > 0 && a->shs != nullptr && a->dL_dsh == nullptr))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "a required backward input or output is NULL");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const GeomLayout GL = GeomLayout::make(a->P);
  const ImageLayout IL = ImageLayout::make(a->W, a->H, stores_state(a->flags));
  if (geom == nullptr || geom_bytes < GL.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "geometry buffer smaller than omnigs_lonlat_geom_bytes(P)");
  if (image == nullptr || image_bytes < IL.total)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "image buffer smaller than omnigs_lonlat_image_bytes_flags(W, H, flags)");
  const int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (binning == nullptr || capacity < 0)
    return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer smaller than omnigs_lonlat_binning_bytes(0)");
  if (int rc = check_aligned(geom, image, binning)) return rc;
  if (a->R > capacity) return fail(OMNIGS_ERR_CAPACITY, "R exceeds the binning buffer's capacity");
  const BinningLayout BL = BinningLayout::make(capacity);
  const int gx = tiles_x(a->W), gy = tiles_y(a->H);
  const int fin = tile_final(a->W, a->H);

  RenderParams r{};
  r.P = a->P;
  r.W = a->W;
  r.H = a->H;
  r.gx = gx;
  r.gy = gy;
  r.ranges = at<uint2>(image, IL.ranges);
  r.point_list = at<uint32_t>(binning, fin ? BL.tvals1 : BL.tvals0);
  r.capacity = capacity;
  r.splat = at<float4>(geom, GL.splat);
  r.color = at<float4>(geom, GL.color);
  r.bg = a->background;
  // NULL per-pixel state: the backward blend recomputes it (transmittance checkpointing)
  r.final_T = IL.store_state ? const_cast<float*>(at<float>(image, IL.final_T)) : nullptr;
  r.n_contrib = IL.store_state ? const_cast<uint32_t*>(at<uint32_t>(image, IL.n_contrib)) : nullptr;
  r.dL_dpix = a->dL_dout_color;
  r.grad_acc = at<float>(geom, GL.grad_acc);
  staged(OMNIGS_STAGE_RENDER_BACKWARD, 1, s, [&] { launch_render_backward(r, s); });
  if (int rc = check_launch("render backward")) return rc;

  PreprocessBackwardParams b{};
  b.P = a->P;
  b.D = a->D;
  b.M = a->M;
  b.W = a->W;
  b.H = a->H;
  b.means3D = a->means3D;
  b.radii = a->radii;
  b.shs = a->shs;
  b.color = at<float4>(geom, GL.color);
  b.splat = at<float4>(geom, GL.splat);
  b.scales = a->scales;
  b.rotations = a->rotations;
  b.cov3D_precomp = a->cov3D_precomp;
  b.scale_modifier = a->scale_modifier;
  b.viewmatrix = a->viewmatrix;
  b.campos = a->campos;
  b.grad_acc = at<float4>(geom, GL.grad_acc);
  b.dL_dmeans2D = a->dL_dmeans2D;
  b.dL_dconic = a->dL_dconic;
  b.dL_dopacity = a->dL_dopacity;
  b.dL_dcolors = a->dL_dcolors;
  b.dL_dmeans3D = a->dL_dmeans3D;
  b.dL_dcov3D = a->dL_dcov3D;
  b.dL_dsh = a->dL_dsh;
  b.dL_dscales = a->dL_dscales;
  b.dL_drotations = a->dL_drotations;
  staged(OMNIGS_STAGE_PREPROCESS_BACKWARD, 1, s, [&] { launch_preprocess_backward(b, s); });
  return check_launch("preprocess backward");
}

int omnigs_mark_visible(int P, const float* means3D, const float* viewmatrix, int camera_type,
                        uint8_t* present, omnigs_stream_t stream) {
  g_last_error.clear();
  if (P < 0) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "P must be >= 0");
  if (camera_type != OMNIGS_CAMERA_LONLAT && camera_type != OMNIGS_CAMERA_PINHOLE)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "[CudaRasterizer]Invalid camera_type");
  if (P == 0) return OMNIGS_OK;
  if (present == nullptr || (camera_type == OMNIGS_CAMERA_PINHOLE && (means3D == nullptr || viewmatrix == nullptr)))
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "present, means3D and viewmatrix are required");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  staged(OMNIGS_STAGE_OTHER, 1, s, [&] {
    launch_mark_visible(P, means3D, viewmatrix, camera_type, reinterpret_cast<bool*>(present), s);
  });
  return check_launch("mark visible");
}

int omnigs_set_blend_batch(int forward, int backward) {
  g_last_error.clear();
  auto ok = [](int b) { return b == 128 || b == 256 || b == 512; };
  if (!ok(forward) || !ok(backward)) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "blend batch sizes must be 128, 256 or 512");
  g_blend_batch[0].store(forward);
  g_blend_batch[1].store(backward);
  return OMNIGS_OK;
}

int omnigs_get_blend_batch(int* forward, int* backward) {
  if (forward) *forward = g_blend_batch[0].load();
  if (backward) *backward = g_blend_batch[1].load();
  return OMNIGS_OK;
}

int omnigs_timing_enable(int enable) {
  std::lock_guard<std::mutex> lock(g_timing_mu);
  g_timing.store(enable != 0);
  return OMNIGS_OK;
}

int omnigs_timing_read(OmnigsStageTimes* out) {
  g_last_error.clear();
  if (out == nullptr) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "out is NULL");
  std::memset(out, 0, sizeof(*out));
  std::lock_guard<std::mutex> lock(g_timing_mu);
  int rc = OMNIGS_OK;
  for (const TimedLaunch& t : g_timed) {
    float ms = 0.f;
    if (cudaEventSynchronize(t.stop) != cudaSuccess || cudaEventElapsedTime(&ms, t.start, t.stop) != cudaSuccess)
      rc = check_launch("timing read");
    out->ms[t.stage] += ms;
    out->launches[t.stage] += (uint64_t)t.kernels;
    g_event_pool.push_back(t.start);
    g_event_pool.push_back(t.stop);
  }
  g_timed.clear();
  return rc;
}

uint64_t omnigs_kernel_launches(void) { return g_launches.load(); }

int omnigs_lonlat_geom_view(const void* geom, int P, OmnigsLonlatGeomView* out) {
  if (geom == nullptr || out == nullptr || P < 0) return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad view arguments");
  const GeomLayout L = GeomLayout::make(P);
  out->splat = at<float>(geom, L.splat);
  out->color = at<float>(geom, L.color);
  out->depth = at<float>(geom, L.depth);
  out->tiles_touched = at<uint32_t>(geom, L.tiles_touched);
  out->depth_order = at<uint32_t>(geom, (kDepthPasses - 1) & 1 ? L.dvals1 : L.dvals0);
  return OMNIGS_OK;
}

int omnigs_lonlat_binning_view(const void* binning, size_t binning_bytes, int W, int H,
                               OmnigsLonlatBinningView* out) {
  if (binning == nullptr || out == nullptr || W <= 0 || H <= 0)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad view arguments");
  const int64_t capacity = BinningLayout::capacity_for(binning_bytes);
  if (capacity < 0) return fail(OMNIGS_ERR_BUFFER_TOO_SMALL, "binning buffer too small");
  const BinningLayout L = BinningLayout::make(capacity);
  const int fin = tile_final(W, H);
  out->tile_ids = at<uint32_t>(binning, fin ? L.tkeys1 : L.tkeys0);
  out->point_list = at<uint32_t>(binning, fin ? L.tvals1 : L.tvals0);
  return OMNIGS_OK;
}

int omnigs_lonlat_image_view(const void* image, int W, int H, OmnigsLonlatImageView* out) {
  if (image == nullptr || out == nullptr || W <= 0 || H <= 0)
    return fail(OMNIGS_ERR_INVALID_ARGUMENT, "bad view arguments");
  const ImageLayout L = ImageLayout::make(W, H);
  out->final_T = at<float>(image, L.final_T);
  out->n_contrib = at<uint32_t>(image, L.n_contrib);
  out->ranges = at<uint32_t>(image, L.ranges);
  return OMNIGS_OK;
}

}  // extern "C"
