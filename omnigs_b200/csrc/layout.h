// Layout of the three opaque state buffers of one lonlat rasterization.
//
// The reference carves GeometryState / ImageState / BinningState out of torch byte tensors
// (cuda_rasterizer/rasterizer_impl.h:37-102).  The buffers stay opaque at the API, so this
// library lays them out for its own kernels:
//
//   geometry (per Gaussian, P):  header | scan look-back u64[scan tiles] |
//                                splat records float4[2P] {x, y, conic a, b}
//                                {conic c, opacity, cull half-width, cull half-height} |
//                                colour float4[P] {r, g, b, clamp bits} | depth f32[P] |
//                                inclusive tile offsets u32[P] | gradient accumulators float4[3P]
//   image (per pixel, N = W*H):  final transmittance f32[N] | last contributor u32[N] |
//                                tile ranges uint2[tiles]
//   binning (per instance, capacity C): keys u64[2][C] | values u32[2][C] |
//                                digit histograms u32[8][256] | sort look-back u32[8][sort tiles][256]
//
// Every array starts on a 256-byte boundary.
#pragma once

#include <cstddef>
#include <cstdint>

namespace omnigs {

constexpr size_t kAlign = 256;
constexpr int kScanBlock = 256;          // Gaussians per preprocess block (one scan tile)
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;           // keys per thread per sort tile
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxSortPasses = 8;        // 64-bit keys
constexpr int64_t kMaxInstances = (int64_t(1) << 30) - 1;  // look-back words hold 30-bit counts

// Device status bits, in GeomHeader::status.
constexpr uint32_t kStatusCapacity = 1u;      // num_rendered exceeded the binning capacity
constexpr uint32_t kStatusLookback = 2u;      // a bounded look-back wait gave up
constexpr uint32_t kStatusOverflow = 4u;      // instance count does not fit the 30-bit counters

struct GeomHeader {
  uint32_t status;
  uint32_t num_rendered;
  uint32_t scan_tile_counter;
  uint32_t pad0;
  uint64_t num_rendered64;
  uint32_t sort_tile_counter[kMaxSortPasses];
  uint32_t reserved[64 - 6 - kMaxSortPasses];
};
static_assert(sizeof(GeomHeader) == 256, "header must be 256 bytes");

__host__ __device__ inline size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

inline int tiles_x(int W) { return (W + 15) / 16; }
inline int tiles_y(int H) { return (H + 15) / 16; }

struct GeomLayout {
  size_t header, scan_state, zero_end, splat, color, depth, offsets, grad_acc, total;
  static GeomLayout make(int64_t P) {
    GeomLayout L;
    size_t o = 0;
    L.header = o; o = align_up(o + sizeof(GeomHeader));
    const int64_t scan_tiles = (P + kScanBlock - 1) / kScanBlock;
    L.scan_state = o; o = align_up(o + sizeof(uint64_t) * scan_tiles);
    L.zero_end = o;  // header and scan state are cleared together before each preprocess
    L.splat = o; o = align_up(o + sizeof(float) * 8 * P);
    L.color = o; o = align_up(o + sizeof(float) * 4 * P);
    L.depth = o; o = align_up(o + sizeof(float) * P);
    L.offsets = o; o = align_up(o + sizeof(uint32_t) * P);
    L.grad_acc = o; o = align_up(o + sizeof(float) * 12 * P);
    L.total = o;
    return L;
  }
};

struct ImageLayout {
  size_t final_T, n_contrib, ranges, total;
  static ImageLayout make(int W, int H) {
    ImageLayout L;
    const int64_t N = (int64_t)W * H;
    const int64_t tiles = (int64_t)tiles_x(W) * tiles_y(H);
    size_t o = 0;
    L.final_T = o; o = align_up(o + sizeof(float) * N);
    L.n_contrib = o; o = align_up(o + sizeof(uint32_t) * N);
    L.ranges = o; o = align_up(o + sizeof(uint32_t) * 2 * tiles);
    L.total = o;
    return L;
  }
};

struct BinningLayout {
  size_t keys0, keys1, vals0, vals1, hist, lookback, total;
  int64_t capacity;
  static int64_t sort_tiles(int64_t capacity) { return (capacity + kSortTile - 1) / kSortTile; }
  static BinningLayout make(int64_t C) {
    BinningLayout L;
    L.capacity = C;
    size_t o = 0;
    L.keys0 = o; o = align_up(o + sizeof(uint64_t) * C);
    L.keys1 = o; o = align_up(o + sizeof(uint64_t) * C);
    L.vals0 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.vals1 = o; o = align_up(o + sizeof(uint32_t) * C);
    L.hist = o; o = align_up(o + sizeof(uint32_t) * kMaxSortPasses * kRadix);
    L.lookback = o; o = align_up(o + sizeof(uint32_t) * kMaxSortPasses * sort_tiles(C) * kRadix);
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

// Number of 8-bit LSD passes that cover key bits [0, 32 + bit), bit = getHigherMsb(tiles)
// (rasterizer_impl.cu:47-62, 651-661).
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

}  // namespace omnigs
