// Layout of the three opaque state buffers of one lonlat rasterization.
//
// The reference carves GeometryState / ImageState / BinningState out of torch byte tensors
// (cuda_rasterizer/rasterizer_impl.h:37-102).  The buffers stay opaque at the API, so this
// library lays them out for its own kernels:
//
//   geometry (per Gaussian, P):  header | duplicate-scan look-back u64[P/256] |
//                                depth-sort look-back u32[4][sort tiles][256] |
//                                splat records float4[2P] {x, y, conic a, b}
//                                {conic c, opacity, cull threshold, conic determinant} |
//                                colour float4[P] {r, g, b, clamp bits} | depth f32[P] |
//                                tiles_touched u32[P] | depth-sort keys/values u32[4][P] |
//                                gradient accumulators float4[3P]
//   image (per pixel, N = W*H):  final transmittance f32[N] | last contributor u32[N] |
//                                tile ranges uint2[tiles]  (tile ranges only with
//                                OMNIGS_FLAG_RECOMPUTE_T: the backward recomputes the rest)
//   binning (per instance, capacity C): tile keys u32[2][C] | Gaussian indices u32[2][C] |
//                                digit histograms u32[7][256] | tile-sort look-back u32[3][tiles][256] |
//                                duplicate emit-block index u32[2][C / 2048 + 1]
//
// Every array starts on a 256-byte boundary.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define OMNIGS_HD __host__ __device__
#else
#define OMNIGS_HD
#endif

namespace omnigs {

constexpr size_t kAlign = 256;
constexpr int kMaxBatchViews = 32;           // views per batched launch
constexpr int kScanBlock = 256;          // threads of a preprocess / duplicate block
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;           // keys per thread per sort tile
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kDepthPasses = 4;          // 32-bit depth keys, 8-bit digits
// The depth sort ping-pongs between two key buffers; with an even pass count its result lands in
// the second, and the duplicate pass uses the first as scratch.
static_assert(kDepthPasses % 2 == 0, "the duplicate pass's scratch is the depth sort's first key buffer");
constexpr int kTilePasses = 3;           // tile ids (<= 21 bits): up to three digits of <= 8 bits
constexpr int kMaxSortPasses = kDepthPasses + kTilePasses;
constexpr int64_t kMaxInstances = (int64_t(1) << 30) - 1;  // look-back words hold 30-bit counts

// Device status bits, in GeomHeader::status.
constexpr uint32_t kStatusCapacity = 1u;      // num_rendered exceeded the binning capacity
constexpr uint32_t kStatusLookback = 2u;      // a bounded look-back wait gave up
constexpr uint32_t kStatusOverflow = 4u;      // instance count does not fit the 30-bit counters
constexpr uint32_t kStatusInconsistent = 8u;  // the duplicate pass counted a different total

struct GeomHeader {
  uint32_t status;
  uint32_t num_rendered;
  uint32_t dup_tile_counter;
  uint32_t pad0;
  unsigned long long num_rendered64;
  uint32_t sort_tile_counter[kMaxSortPasses];
  uint32_t reserved[64 - 6 - kMaxSortPasses];
};
static_assert(sizeof(GeomHeader) == 256, "header must be 256 bytes");

OMNIGS_HD inline size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

inline int tiles_x(int W) { return (W + 15) / 16; }
inline int tiles_y(int H) { return (H + 15) / 16; }
inline int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }

struct GeomLayout {
  size_t header, dup_scan, depth_lookback, zero_end, splat, color, depth, tiles_touched, dkeys0,
      dkeys1, dvals0, dvals1, grad_acc, total;
  static GeomLayout make(int64_t P) {
    GeomLayout L;
    size_t o = 0;
    L.header = o; o = align_up(o + sizeof(GeomHeader));
    L.dup_scan = o; o = align_up(o + sizeof(uint64_t) * ((P + kScanBlock - 1) / kScanBlock));
    L.depth_lookback = o; o = align_up(o + sizeof(uint32_t) * kDepthPasses * sort_tiles(P) * kRadix);
    L.zero_end = o;  // everything above is cleared before each preprocess
    L.splat = o; o = align_up(o + sizeof(float) * 8 * P);
    L.color = o; o = align_up(o + sizeof(float) * 4 * P);
    L.depth = o; o = align_up(o + sizeof(float) * P);
    L.tiles_touched = o; o = align_up(o + sizeof(uint32_t) * P);
    L.dkeys0 = o; o = align_up(o + sizeof(uint32_t) * P);
    L.dkeys1 = o; o = align_up(o + sizeof(uint32_t) * P);
    L.dvals0 = o; o = align_up(o + sizeof(uint32_t) * P);
    L.dvals1 = o; o = align_up(o + sizeof(uint32_t) * P);
    L.grad_acc = o; o = align_up(o + sizeof(float) * 12 * P);
    L.total = o;
    return L;
  }
};

// With store_state false (transmittance checkpointing) the buffer holds only the tile ranges.
struct ImageLayout {
  size_t final_T, n_contrib, ranges, total;
  bool store_state;
  static ImageLayout make(int W, int H, bool store_state = true) {
    ImageLayout L;
    const int64_t N = store_state ? (int64_t)W * H : 0;
    const int64_t tiles = (int64_t)tiles_x(W) * tiles_y(H);
    size_t o = 0;
    L.store_state = store_state;
    L.final_T = o; o = align_up(o + sizeof(float) * N);
    L.n_contrib = o; o = align_up(o + sizeof(uint32_t) * N);
    L.ranges = o; o = align_up(o + sizeof(uint32_t) * 2 * tiles);
    L.total = o;
    return L;
  }
};

// The duplicate pass writes the instance list in blocks of kEmitBlock instances; its scan records,
// per such block, the depth-order positions of the Gaussians holding the block's first and last
// instance (emit_first / emit_last).
constexpr int kEmitBlock = 2048;
inline int64_t emit_blocks(int64_t capacity) { return (capacity + kEmitBlock - 1) / kEmitBlock; }
// Gaussians per block of the duplicate's scan (4 per thread)
constexpr int kScanTile = 1024;

struct BinningLayout {
  size_t tkeys0, tkeys1, tvals0, tvals1, hist, tile_lookback, emit_first, emit_last, total;
  int64_t capacity;
  static BinningLayout make(int64_t C) {
    BinningLayout L;
    L.capacity = C;
    size_t o = 0;
    L.tkeys0 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.tkeys1 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.tvals0 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.tvals1 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.hist = o; o = align_up(o + sizeof(uint32_t) * kMaxSortPasses * kRadix);
    // room for a per-view tile sort of a batch: up to kMaxBatchViews more (partial) tiles per pass
    L.tile_lookback = o; o = align_up(o + sizeof(uint32_t) * kTilePasses * (sort_tiles(C) + kMaxBatchViews) * kRadix);
    L.emit_first = o; o = align_up(o + sizeof(uint32_t) * (emit_blocks(C) + 1));
    L.emit_last = o; o = align_up(o + sizeof(uint32_t) * (emit_blocks(C) + 1));
    L.total = o;
    return L;
  }
  // Largest capacity whose layout fits in `bytes`.
  static int64_t capacity_for(size_t bytes) {
    if (bytes < make(0).total) return -1;
    int64_t lo = 0, hi = int64_t(1) << 31;
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo + 1) / 2;
      if (make(mid).total <= bytes)
        lo = mid;
      else
        hi = mid - 1;
    }
    return lo;
  }
};

// State of a batch of V views over P shared Gaussians (one buffer; the instance lists use a
// BinningLayout buffer as in the single-view case).  Per-(view, Gaussian) arrays are view-major;
// per-pixel arrays hold the views' pixels back to back, ranges the views' tiles back to back.
//
//   header | instances per view u64[32] | view tile bases u32[32] | duplicate-scan look-back u64[VP/256] |
//   depth-sort look-back u32[4][V sort tiles(P)][256] | depth histograms u32[V][4][256] |
//   tile-sort histograms u32[V][3][256] |
//   radii i32[VP] | splat records float4[2VP] | colour float4[VP] | depth f32[VP] |
//   depth-sort keys/values u32[4][VP] | gradient accumulators float4[3VP] |
//   final transmittance f32[pixels] | last contributor u32[pixels] | tile ranges uint2[tiles]
struct BatchLayout {
  size_t header, view_rendered, view_key_base, dup_scan, depth_lookback, depth_hist, tile_hist, zero_end, radii, splat, color, depth,
      dkeys0, dkeys1, dvals0, dvals1, grad_acc, final_T, n_contrib, ranges, total;
  static BatchLayout make(int64_t P, int V, int64_t pixels, int64_t tiles) {
    BatchLayout L;
    const int64_t R = P * V;
    size_t o = 0;
    L.header = o; o = align_up(o + sizeof(GeomHeader));
    // the view tile bases directly follow the per-view counts: the tile sort finds them there
    static_assert(sizeof(uint64_t) * kMaxBatchViews % kAlign == 0, "view_key_base must follow view_rendered");
    L.view_rendered = o; o = align_up(o + sizeof(uint64_t) * kMaxBatchViews);
    L.view_key_base = o; o = align_up(o + sizeof(uint32_t) * kMaxBatchViews);
    L.dup_scan = o; o = align_up(o + sizeof(uint64_t) * ((R + kScanBlock - 1) / kScanBlock));
    L.depth_lookback = o; o = align_up(o + sizeof(uint32_t) * kDepthPasses * sort_tiles(P) * V * kRadix);
    L.depth_hist = o; o = align_up(o + sizeof(uint32_t) * V * kDepthPasses * kRadix);
    L.tile_hist = o; o = align_up(o + sizeof(uint32_t) * V * kTilePasses * kRadix);
    L.zero_end = o;  // everything above is cleared before each pass
    L.radii = o; o = align_up(o + sizeof(int32_t) * R);
    L.splat = o; o = align_up(o + sizeof(float) * 8 * R);
    L.color = o; o = align_up(o + sizeof(float) * 4 * R);
    L.depth = o; o = align_up(o + sizeof(float) * R);
    L.dkeys0 = o; o = align_up(o + sizeof(uint32_t) * R);
    L.dkeys1 = o; o = align_up(o + sizeof(uint32_t) * R);
    L.dvals0 = o; o = align_up(o + sizeof(uint32_t) * R);
    L.dvals1 = o; o = align_up(o + sizeof(uint32_t) * R);
    L.grad_acc = o; o = align_up(o + sizeof(float) * 12 * R);
    L.final_T = o; o = align_up(o + sizeof(float) * pixels);
    L.n_contrib = o; o = align_up(o + sizeof(uint32_t) * pixels);
    L.ranges = o; o = align_up(o + sizeof(uint32_t) * 2 * tiles);
    L.total = o;
    return L;
  }
};

// getHigherMsb (rasterizer_impl.cu:47-62): the reference sorts key bits [0, 32 + bit), i.e. all
// tile-id bits; the tile passes here cover the same `bit` bits (rasterizer_impl.cu:651-661).
inline uint32_t higher_msb(uint32_t n);

// Digits of the tile sort: `bit` tile-id bits split into passes of at most 8 bits.
struct TileDigits {
  int passes;
  int shift[kTilePasses];
  uint32_t mask[kTilePasses];
  static TileDigits make(int W, int H);
  static TileDigits from_tiles(uint32_t tiles);
};

inline uint32_t higher_msb(uint32_t n) {
  uint32_t msb = sizeof(n) * 4;
  uint32_t step = msb;
  while (step > 1) {
    step /= 2;
    if (n >> msb)
      msb += step;
    else
      msb -= step;
  }
  if (n >> msb) msb++;
  return msb;
}

inline TileDigits TileDigits::make(int W, int H) {
  return from_tiles((uint32_t)tiles_x(W) * (uint32_t)tiles_y(H));
}

inline TileDigits TileDigits::from_tiles(uint32_t tiles) {
  const int bit = (int)higher_msb(tiles);
  TileDigits t{};
  t.passes = (bit + kRadixBits - 1) / kRadixBits;
  if (t.passes < 1) t.passes = 1;
  int shift = 0;
  for (int i = 0; i < t.passes; ++i) {
    const int width = (bit - shift + (t.passes - i) - 1) / (t.passes - i);  // spread evenly
    t.shift[i] = shift;
    t.mask[i] = width >= 32 ? 0xffffffffu : ((1u << width) - 1u);
    shift += width;
  }
  return t;
}

}  // namespace omnigs
