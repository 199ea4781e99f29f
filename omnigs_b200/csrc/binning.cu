// Binning: the reference's sorted instance list and tile ranges (rasterizer_impl.cu:94-167,
// 622-679) from a depth sort of the Gaussians plus a tile sort of the instances.
//
// The reference emits one (tile << 32 | depth_bits) key per (Gaussian, tile) pair in Gaussian
// order and sorts them with a stable LSD radix sort over bits [0, 32 + getHigherMsb(tiles)).  The
// result is fully determined: instances ordered by tile, then by depth bits, then -- a Gaussian
// appears at most once per tile and the list starts in Gaussian order -- by Gaussian index.  The
// same order is produced here with far fewer passes over the instances:
//  1. depth sort: a stable LSD radix sort (4 onesweep passes of 8 bits) of the P Gaussians by the
//     bits of their depth, i.e. the order (depth bits, index);
//  2. duplicate: a scan of the Gaussians' tile counts in that order (decoupled look-back), then
//     a load-balanced emission of the instances in that order (every block writes the same number
//     of instances), counting the digits of the keys it writes for the tile sort;
//  3. tile sort: a stable LSD radix sort (2 onesweep passes) of the instances by tile id only
//     (for a batch of views, per view on view-local tile ids when those need fewer passes than
//     the batch's global ids: each view's instances are contiguous after step 2).
// Stability makes (1)+(3) equal to the reference's single sort: instance passes drop from six
// over 12-byte items to two over 8-byte items; the four depth passes run over P, not R, items.
//  4. ranges: per-tile [start, end) over the sorted tile ids.
// Counts live on the device: every kernel reads num_rendered from the geometry header and does no
// work if it exceeds the binning capacity.  Waits on other blocks are bounded.
#include <algorithm>

#include "device_util.cuh"
#include "kernels.h"
#include "lonlat_math.cuh"

namespace omnigs {
namespace {

constexpr uint32_t kLbAggregate = 1u << 30;
constexpr uint32_t kLbPrefix = 2u << 30;
constexpr uint32_t kLbValue = (1u << 30) - 1;
constexpr unsigned long long kScanAggregate = 1ull << 62;
constexpr unsigned long long kScanPrefix = 2ull << 62;
constexpr unsigned long long kScanValue = (1ull << 62) - 1;
// Predecessors a look-back reads per round.  Measured on a B200 (1M Gaussians, 2048x1024): 16 or
// 32 per round made every sort pass slower (depth passes 21 -> 24-27 us, tile passes 90 -> 95-125
// us), so the walk is not bound by its round trips.  Nor is the pass bound by its look-back: a
// reduce-then-scan in its place (a kernel counting every tile's digits and scanning the counts
// over the tiles, then the pass without waits) made the sort slower, 0.294 -> 0.366 ms per view:
// the count kernels took 12-27 us each and the passes got only 4-10 us faster.
constexpr int kLookbackBatch = 8;

__device__ __forceinline__ bool instances_fit(const GeomHeader* hdr, int64_t capacity) {
  return (hdr->status & kStatusOverflow) == 0 && hdr->num_rendered64 <= (unsigned long long)capacity;
}

// Element count of a sort/histogram: a host value, or the device num_rendered (0 if it does not
// fit the capacity, in which case the duplicate pass has flagged the overflow).
__device__ __forceinline__ uint32_t item_count(const GeomHeader* count_hdr, uint32_t n_host, int64_t capacity) {
  if (count_hdr == nullptr) return n_host;
  return instances_fit(count_hdr, capacity) ? count_hdr->num_rendered : 0u;
}

// ---------------------------------------------------------------- digit histograms ------------
// Adds the warp's digits (lanes in `live`, a prefix of the warp) to a shared histogram.  Keys of a
// sort are either spread over many digits (per-lane atomics rarely collide) or nearly constant
// within a warp (the top digit of depth bits): when every live lane holds lane 0's digit, lane 0
// adds the whole count with one atomic.
__device__ __forceinline__ void count_digit(uint32_t* hist, uint32_t digit, bool valid, unsigned live, int lane) {
  const uint32_t d0 = __shfl_sync(kFullMask, digit, 0);
  if (__all_sync(kFullMask, !valid || digit == d0)) {
    if (lane == 0 && live) atomicAdd(&hist[d0], (uint32_t)__popc(live));
  } else if (valid) {
    atomicAdd(&hist[digit], 1u);
  }
}

constexpr int kHistUnroll = 4;  // keys per thread loaded before any of them is counted

__global__ void __launch_bounds__(256) histogram_kernel(const __grid_constant__ HistParams p) {
  __shared__ uint32_t s_hist[kDepthPasses][kRadix];
  for (int i = threadIdx.x; i < kDepthPasses * kRadix; i += blockDim.x) (&s_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = p.seg_len ? p.seg_len : item_count(p.count_hdr, p.n_host, p.capacity);
  const size_t seg_base = (size_t)blockIdx.y * n;  // gridDim.y segments
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  // Whole warps iterate together (the counting votes over the warp); each thread first loads
  // kHistUnroll keys (independent loads in flight), then counts them.
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride * kHistUnroll) {
    uint32_t key[kHistUnroll];
    bool valid[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) {
      const uint32_t i = base + u * stride + lane;
      valid[u] = i < n;
      key[u] = valid[u] ? p.keys[seg_base + i] : 0u;
    }
    unsigned live[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) live[u] = __ballot_sync(kFullMask, valid[u]);
#pragma unroll
    for (int q = 0; q < kDepthPasses; ++q) {
      if (q >= p.passes) break;
#pragma unroll
      for (int u = 0; u < kHistUnroll; ++u)
        count_digit(s_hist[q], (key[u] >> p.shift[q]) & p.mask[q], valid[u], live[u], lane);
    }
  }
  __syncthreads();
  uint32_t* hist = p.hist + (size_t)blockIdx.y * p.passes * kRadix;
  for (int i = threadIdx.x; i < p.passes * kRadix; i += blockDim.x) {
    const uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

// ---------------------------------------------------------------- onesweep pass ---------------
template <int kTile>
struct SortSmem {
  uint32_t warp_hist[kSortThreads / 32][kRadix];
  uint32_t block_excl[kRadix];
  uint32_t global_base[kRadix];
  uint32_t scan_tmp[kSortThreads / 32];
  uint32_t tile;
  uint32_t pad[3];
  uint32_t keys[kTile];
  uint32_t vals[kTile];
  // the block's segment as thread 0 resolved it (variable segments): index (num_segs: none), item
  // count, tile within the segment, first item, key base
  uint32_t seg, seg_n, seg_tile, seg_first, seg_key_base;
};

// Exclusive scan of one value per thread across the block (kSortThreads == kRadix == 256).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scan_tmp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t n = __shfl_up_sync(kFullMask, x, o);
    if (lane >= o) x += n;
  }
  if (lane == 31) scan_tmp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < kSortThreads / 32) ? scan_tmp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < kSortThreads / 32; o <<= 1) {
      const uint32_t n = __shfl_up_sync(kFullMask, w, o);
      if (lane >= o) w += n;
    }
    if (lane < kSortThreads / 32) scan_tmp[lane] = w;
  }
  __syncthreads();
  total = scan_tmp[kSortThreads / 32 - 1];
  const uint32_t r = x - v + (warp > 0 ? scan_tmp[warp - 1] : 0u);
  __syncthreads();
  return r;
}

// One stable LSD pass over (u32 key, u32 value) pairs on the digit (key >> shift) & mask.  A block
// ranks a 4096-item tile in shared memory (warp multi-split from per-bit ballots: equal digits keep
// their input order), publishes its per-digit counts, resolves its global digit offsets by
// decoupled look-back (tiles are taken in launch order from an atomic counter, so a block only
// waits on blocks that are already running) and writes runs of equal digits coalesced.  In a
// segmented sort every segment is an independent sort whose look-back chain starts at the
// segment's first tile (segments of equal length, or of device-side lengths, whose keys are then
// segment-local and get seg_key_base added back in the last pass); a value-less first pass numbers
// items by their global index.
// Launches of this pass measured ~2 us slower each on a B200 with a 136-byte parameter block than
// with a 128-byte one.
static_assert(sizeof(OnesweepParams) <= 128, "keep the onesweep parameter block at 128 bytes or less");

// Tiles of kSortTile keys, 16 per thread.  Measured on a B200: 1024-key tiles (4 per thread, five
// blocks per SM) made the depth passes over 1M Gaussians slower, 22 -> 30 us each (4x the blocks,
// look-back chains and per-tile scans), so every pass uses the 4096-key tiles.
template <bool kVarSeg>
__global__ void __launch_bounds__(kSortThreads, 3) onesweep_kernel(OnesweepParams p) {
  constexpr int kItems = kSortItems;
  constexpr int kTile = kSortTile;
  __shared__ SortSmem<kTile> sm;
  uint32_t n = 0, tiles_per_seg = 1, ntiles = 0;
  if (!kVarSeg) {
    n = p.seg_len ? p.seg_len : item_count(p.count_hdr, p.n_host, p.capacity);
    tiles_per_seg = (n + kTile - 1) / kTile;
    ntiles = tiles_per_seg * (p.seg_len ? p.num_segs : 1u);
  }
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(p.tile_counter, 1u);
    sm.tile = t;
    if (kVarSeg) {  // variable segments: tickets run over the segments' tiles in order
      const bool fit = instances_fit(p.count_hdr, p.capacity);
      uint32_t first_tile = 0, first_item = 0;
      sm.seg = p.num_segs;
      for (uint32_t sg = 0; sg < p.num_segs; ++sg) {
        const uint32_t ns = fit ? (uint32_t)p.seg_counts[sg] : 0u;
        const uint32_t ts = (ns + kTile - 1) / kTile;
        if (t < first_tile + ts) {
          sm.seg = sg;
          sm.seg_n = ns;
          sm.seg_tile = t - first_tile;
          sm.seg_first = first_item;
          sm.seg_key_base = reinterpret_cast<const uint32_t*>(p.seg_counts + kMaxBatchViews)[sg];
          break;
        }
        first_tile += ts;
        first_item += ns;
      }
    }
  }
  for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&sm.warp_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t ticket = sm.tile;
  // this block's segment, its item count and first item, and the tile index within it
  uint32_t seg, tile;
  size_t seg_base;
  if (kVarSeg) {
    seg = sm.seg;
    if (seg >= p.num_segs) return;
    n = sm.seg_n;
    tile = sm.seg_tile;
    seg_base = sm.seg_first;
  } else {
    if (ticket >= ntiles) return;
    seg = ticket / tiles_per_seg;
    tile = ticket - seg * tiles_per_seg;  // tile index within the segment
    seg_base = (size_t)seg * n;
  }
  const uint32_t* keys_in = p.keys_in + seg_base;
  const uint32_t* vals_in = p.vals_in ? p.vals_in + seg_base : nullptr;
  uint32_t* keys_out = p.keys_out + seg_base;
  uint32_t* vals_out = p.vals_out + seg_base;
  const uint32_t* hist = p.hist + (size_t)seg * p.hist_seg_stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const uint32_t mask = p.mask;
  const int shift = p.shift;

  // load the whole tile first (independent loads in flight), then rank
  uint32_t key[kItems], val[kItems];
  const uint32_t tile_base = tile * kTile + warp * (kItems * 32) + lane;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const uint32_t idx = tile_base + k * 32;
    key[k] = idx < n ? keys_in[idx] : 0xffffffffu;
  }
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const uint32_t idx = tile_base + k * 32;
    val[k] = idx < n ? (vals_in ? vals_in[idx] : (uint32_t)(seg_base + idx)) : 0u;
  }
  // where each digit starts in the whole output
  uint32_t unused;
  sm.global_base[threadIdx.x] = block_exclusive_scan(hist[threadIdx.x], sm.scan_tmp, unused);

  uint32_t rank[kItems];
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const bool valid = tile_base + k * 32 < n;
    const uint32_t digit = (key[k] >> shift) & mask;
    // the valid lanes holding the same digit: one ballot per digit bit (measured faster on a B200
    // than match.any: depth passes 21 -> 18 us, tile passes 86-96 -> 80 us at 1M Gaussians)
    unsigned peers = __ballot_sync(kFullMask, valid);
#pragma unroll
    for (int b = 0; b < kRadixBits; ++b) {
      const bool bit = (digit >> b) & 1u;
      const unsigned bal = __ballot_sync(kFullMask, bit);
      peers &= bit ? bal : ~bal;
    }
    if (!valid) peers = 1u << lane;
    const int leader = __ffs(peers) - 1;
    // every lane reads its digit's running count; the digit's first lane then advances it
    const uint32_t old = valid ? sm.warp_hist[warp][digit] : 0u;
    __syncwarp();
    if (valid && lane == leader) sm.warp_hist[warp][digit] = old + __popc(peers);
    __syncwarp();
    rank[k] = valid ? (old + __popc(peers & lt_mask)) : 0xffffffffu;
  }
  __syncthreads();

  // per digit: exclusive offsets of each warp, block count, block-local digit start
  const int d = threadIdx.x;
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < kSortThreads / 32; ++w) {
    const uint32_t t = sm.warp_hist[w][d];
    sm.warp_hist[w][d] = run;
    run += t;
  }
  const uint32_t count = run;
  uint32_t tile_items;
  sm.block_excl[d] = block_exclusive_scan(count, sm.scan_tmp, tile_items);
  __syncthreads();  // every digit's block-local start is read by other threads below

  // decoupled look-back for digit d (digits above the mask are empty everywhere)
  uint32_t* lb = p.lookback + (size_t)(ticket - tile) * kRadix;  // this segment's chain
  if (tile == 0 || (uint32_t)d > mask) {
    st_relaxed_u32(&lb[(size_t)tile * kRadix + d], kLbPrefix | count);
  } else {
    st_relaxed_u32(&lb[(size_t)tile * kRadix + d], kLbAggregate | count);
    uint32_t prev = 0;
    int64_t j = (int64_t)tile - 1;
    bool gave_up = false, found = false;
    while (!found) {
      uint32_t w[kLookbackBatch];
#pragma unroll
      for (int b = 0; b < kLookbackBatch; ++b)
        w[b] = (j - b >= 0) ? ld_relaxed_u32(&lb[(size_t)(j - b) * kRadix + d]) : kLbPrefix;
#pragma unroll
      for (int b = 0; b < kLookbackBatch; ++b) {
        uint32_t x = w[b];
        if (!found && (x >> 30) == 0) {
          int spins = 0;
          do {
            if (++spins > kMaxSpins) {
              gave_up = true;
              x = kLbPrefix;
              break;
            }
            __nanosleep(32);
            x = ld_relaxed_u32(&lb[(size_t)(j - b) * kRadix + d]);
          } while ((x >> 30) == 0);
        }
        if (!found) {
          prev += x & kLbValue;
          found = (x >> 30) == 2;
        }
      }
      j -= kLookbackBatch;
    }
    if (gave_up) atomicOr(&p.hdr->status, kStatusLookback);
    st_relaxed_u32(&lb[(size_t)tile * kRadix + d], kLbPrefix | ((prev + count) & kLbValue));
    sm.global_base[d] += prev;
  }

  // reorder the tile in shared memory by digit
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    if (rank[k] != 0xffffffffu) {
      const uint32_t digit = (key[k] >> shift) & mask;
      const uint32_t pos = sm.block_excl[digit] + sm.warp_hist[warp][digit] + rank[k];
      if (pos < (uint32_t)kTile) {  // always true: ranks are consistent within the block
        sm.keys[pos] = key[k];
        sm.vals[pos] = val[k];
      }
    }
  }
  __syncthreads();
  // the last pass of a variable-segment sort turns segment-local keys back into global ones
  const uint32_t key_add = (kVarSeg && p.add_key_base) ? sm.seg_key_base : 0u;
  for (uint32_t i = threadIdx.x; i < tile_items; i += kSortThreads) {
    const uint32_t k32 = sm.keys[i];
    const uint32_t digit = (k32 >> shift) & mask;
    const uint32_t out = sm.global_base[digit] + (i - sm.block_excl[digit]);
    if (out < n) {  // always true unless a look-back gave up (the status word then says so)
      keys_out[out] = k32 + key_add;
      vals_out[out] = sm.vals[i];
    }
  }
}

// ---------------------------------------------------------------- duplicate -------------------
// duplicateWithKeys (rasterizer_impl.cu:94-140) over the depth-sorted Gaussians, in two kernels:
//  1. instance_scan_kernel: the inclusive scan of the Gaussians' tile counts in depth order (block
//     b takes sorted positions [1024 b, 1024 b + 1024), four per thread: block scan plus a
//     decoupled look-back over the preceding blocks), written to p.incl; every Gaussian whose
//     instances hold the first or last instance of an emit block (kEmitBlock instances) records
//     its position there (p.emit_first / p.emit_last);
//  2. instance_emit_kernel: block b writes instances [2048 b, 2048 b + 2048) of the list: every
//     block does the same amount of work however the instances are spread over the Gaussians
//     (the nearest splats, first in depth order, cover thousands of tiles each).  It stages the
//     offsets and tile rects of its Gaussians in shared memory; each thread writes 8 consecutive
//     instances (one binary search for the first one's Gaussian, then a walk through the rect and
//     on to the next Gaussians, two 16-byte stores per array) and counts the digit histograms of
//     the tile sort that follows.
// One kernel doing both measured ~150 us at 400k and 1M Gaussians alike: a block's warps each
// emitted their own Gaussians' instances, so a block held its SM slots until its busiest warp was
// done (62 % of the stall samples were barrier waits).

// Tile rect of record `rec` (view `view`) in the duplicate's terms: instance count, rect width,
// first column, tile-id pitch and the id of the rect's first row (view-local when per view).
struct RecordRect {
  uint32_t count, row_origin;
  int pitch, width, col0;
};

template <bool kPerView>
__device__ __forceinline__ RecordRect record_rect(const DuplicateParams& p, uint32_t rec, uint32_t view) {
  RecordRect r;
  r.count = 0;
  r.row_origin = 0;
  r.pitch = 1;
  r.width = 1;
  r.col0 = 0;
  const int radius = (rec - view * (uint32_t)p.P < (uint32_t)p.P) ? p.radii[rec] : 0;
  if (radius > 0) {
    const float4 a = p.splat[2 * rec];
    const int gx = p.gx[view];
    int2 rmin, rmax;
    if (p.seam_wrap)
      tile_rect_cyclic(make_float2(a.x, a.y), radius, gx, p.gy[view], rmin, rmax);
    else
      tile_rect(make_float2(a.x, a.y), radius, gx, p.gy[view], rmin, rmax);
    r.width = rmax.x - rmin.x;
    r.count = (uint32_t)r.width * (uint32_t)(rmax.y - rmin.y);
    if (r.count == 0) r.width = 1;
    r.pitch = gx;
    r.col0 = rmin.x;
    // per-view counting writes view-local tile ids (the tile sort restores the global ids)
    r.row_origin = (kPerView ? 0u : p.tile_base[view]) + (uint32_t)rmin.y * (uint32_t)gx;
  }
  return r;
}

__device__ __forceinline__ uint32_t record_view(const DuplicateParams& p, uint32_t i) {
  return (p.V == 1) ? 0u : i / (uint32_t)p.P;  // the depth order keeps records in their view
}

constexpr int kScanItems = kScanTile / kScanBlock;  // Gaussians per scan thread

template <bool kPerView>
__global__ void __launch_bounds__(kScanBlock) instance_scan_kernel(const __grid_constant__ DuplicateParams p) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanBlock / 32];
  __shared__ unsigned long long s_excl;
  if (!instances_fit(p.hdr, p.capacity)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&p.hdr->status, kStatusCapacity);
    return;
  }
  if (kPerView && blockIdx.x == 0 && threadIdx.x < p.V) p.key_base_out[threadIdx.x] = p.tile_base[threadIdx.x];
  if (threadIdx.x == 0) s_tile = atomicAdd(&p.hdr->dup_tile_counter, 1u) + p.skip_tiles;
  __syncthreads();
  const uint32_t tile = s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t items = (uint32_t)p.P * (uint32_t)p.V;
  const uint32_t i0 = tile * (uint32_t)kScanTile + threadIdx.x * (uint32_t)kScanItems;
  uint32_t cnt[kScanItems];
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    const uint32_t i = i0 + u;
    cnt[u] = 0;
    if (i < items) {
      const RecordRect r = record_rect<kPerView>(p, p.order[i], record_view(p, i));
      cnt[u] = r.count;
      p.rect_row[i] = r.row_origin;
      p.rect_cw[i] = ((uint32_t)r.col0 & 0xffffu) | ((uint32_t)r.width << 16);
    }
  }
  uint32_t thread_total = 0;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) thread_total += cnt[u];
  // block inclusive scan of the thread totals
  uint32_t v = thread_total;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t n = __shfl_up_sync(kFullMask, v, o);
    if (lane >= o) v += n;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = (lane < kScanBlock / 32) ? s_warp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < kScanBlock / 32; o <<= 1) {
      const uint32_t n = __shfl_up_sync(kFullMask, w, o);
      if (lane >= o) w += n;
    }
    if (lane < kScanBlock / 32) s_warp[lane] = w;
  }
  __syncthreads();
  const uint32_t thread_excl = v - thread_total + (warp > 0 ? s_warp[warp - 1] : 0u);
  const unsigned long long block_total = s_warp[kScanBlock / 32 - 1];
  // decoupled look-back across blocks (warp 0)
  if (warp == 0) {
    if (tile == 0) {
      if (lane == 0) {
        st_relaxed_u64(&p.scan_state[0], kScanPrefix | block_total);
        s_excl = 0;
      }
    } else {
      if (lane == 0) st_relaxed_u64(&p.scan_state[tile], kScanAggregate | block_total);
      unsigned long long excl = 0;
      long long base = (long long)tile - 1;
      bool gave_up = false;
      const int max_spins = p.max_spins > 0 ? p.max_spins : kMaxSpins;
      for (;;) {
        const long long j = base - lane;
        unsigned long long w = kScanPrefix;  // virtual zero prefix before the first block
        if (j >= 0) {
          w = ld_relaxed_u64(&p.scan_state[j]);
          int spins = 0;
          while ((w >> 62) == 0) {
            if (++spins > max_spins) {
              gave_up = true;
              w = kScanPrefix;
              break;
            }
            __nanosleep(64);
            w = ld_relaxed_u64(&p.scan_state[j]);
          }
        }
        const unsigned prefix_lanes = __ballot_sync(kFullMask, (w >> 62) == 2);
        const int stop = prefix_lanes ? (__ffs(prefix_lanes) - 1) : 31;
        unsigned long long c = (lane <= stop) ? (w & kScanValue) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFullMask, c, o);
        excl += c;
        if (prefix_lanes) break;
        base -= 32;
      }
      if (__any_sync(kFullMask, gave_up) && lane == 0) atomicOr(&p.hdr->status, kStatusLookback);
      if (lane == 0) {
        st_relaxed_u64(&p.scan_state[tile], kScanPrefix | ((excl + block_total) & kScanValue));
        s_excl = excl;
      }
    }
  }
  __syncthreads();
  const unsigned long long R = p.hdr->num_rendered64;
  const uint32_t nblocks = (uint32_t)((R + kEmitBlock - 1) / kEmitBlock);  // emit blocks (R fits the capacity)
  unsigned long long incl = s_excl + thread_excl;
#pragma unroll
  for (int u = 0; u < kScanItems; ++u) {
    const uint32_t i = i0 + u;
    const unsigned long long start = incl;
    incl += cnt[u];
    if (i >= items) continue;
    p.incl[i] = (uint32_t)min(incl, 0xffffffffull);
    if (cnt[u] == 0 || incl > R) continue;  // (past R only when the scan is inconsistent)
    // the emit blocks whose first instance (b * kEmitBlock) lies in [start, incl)
    for (unsigned long long b = (start + kEmitBlock - 1) / kEmitBlock; b * kEmitBlock < incl && b < nblocks; ++b)
      p.emit_first[b] = i;
    // ... and whose last instance (min((b + 1) kEmitBlock, R) - 1) does
    for (unsigned long long b = start / kEmitBlock; b < nblocks && b * kEmitBlock < incl; ++b) {
      const unsigned long long last = min((b + 1) * (unsigned long long)kEmitBlock, R) - 1;
      if (last >= start && last < incl) p.emit_last[b] = i;
    }
  }
  const uint32_t last_tile = (items + kScanTile - 1) / kScanTile - 1u;
  if (tile == last_tile && threadIdx.x == kScanBlock - 1 && s_excl + block_total != R)
    atomicOr(&p.hdr->status, kStatusInconsistent);
}

constexpr int kEmitPerThread = kEmitBlock / kScanBlock;
constexpr int kEmitStage = 1025;  // Gaussians of a block staged in shared memory (more: read from global memory)

__device__ __forceinline__ float rcp_approx_f(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <bool kPerView>
__global__ void __launch_bounds__(kScanBlock) instance_emit_kernel(const __grid_constant__ DuplicateParams p) {
  // digit counts of the tile sort: [slot][pass][digit], slot = view - (the block's first view)
  // when counted per view; views past kSlots (a block spanning many small views) count directly
  // into the global histogram
  constexpr int kHistSlot = kTilePasses * kRadix;
  constexpr int kSlots = kPerView ? 2 : 1;
  __shared__ uint32_t s_hist[kSlots * kHistSlot];
  // the block's Gaussians: inclusive offset, record, first row's tile id, first column | width,
  // tile-id pitch | view
  __shared__ uint32_t s_incl[kEmitStage], s_rec[kEmitStage], s_row[kEmitStage], s_cw[kEmitStage], s_pv[kEmitStage];
  if (!instances_fit(p.hdr, p.capacity)) return;  // the scan kernel has flagged the overflow
  const uint32_t R = p.hdr->num_rendered;
  const uint32_t o_lo = blockIdx.x * (uint32_t)kEmitBlock;
  if (o_lo >= R) return;
  const uint32_t o_hi = min(R, o_lo + (uint32_t)kEmitBlock);  // exclusive (R <= capacity)
  const int lane = threadIdx.x & 31;
  const uint32_t items = (uint32_t)p.P * (uint32_t)p.V;
  for (int k = threadIdx.x; k < kSlots * kHistSlot; k += kScanBlock) s_hist[k] = 0;
  // (both clamped: after an inconsistent scan, which the status word reports, the entries may be
  // stale; the reads stay in range)
  const uint32_t g_first = min(p.emit_first[blockIdx.x], items - 1u);
  const uint32_t g_last = min(p.emit_last[blockIdx.x], items - 1u);
  const uint32_t n = g_last >= g_first ? g_last - g_first + 1u : 1u;
  // Gaussians between g_first and g_last with no instances (culled views' records) can make the
  // range longer than the block's instance count: then offsets and rects are read from global memory
  const bool staged = n <= (uint32_t)kEmitStage;
  if (staged)
    for (uint32_t t = threadIdx.x; t < n; t += kScanBlock) {
      const uint32_t i = g_first + t;
      const uint32_t view = record_view(p, i);
      s_incl[t] = p.incl[i];
      s_rec[t] = p.order[i];
      s_row[t] = p.rect_row[i];
      s_cw[t] = p.rect_cw[i];
      s_pv[t] = (uint32_t)p.gx[view] | (view << 16);
    }
  __syncthreads();
  const uint32_t* incl = staged ? s_incl : p.incl + g_first;
  const uint32_t excl0 = g_first > 0 ? p.incl[g_first - 1] : 0u;
  const uint32_t view0 = record_view(p, g_first);
  // Thread t writes the kEmitPerThread consecutive instances from o0: one binary search finds the
  // Gaussian of the first, the others step through the rect (or on to the next Gaussians with
  // instances, whose first instance they then are) without a search or a division.
  const uint32_t o0 = o_lo + (uint32_t)threadIdx.x * (uint32_t)kEmitPerThread;
  uint32_t j = 0;  // the first of the block's Gaussians whose inclusive offset exceeds o0
  {
    uint32_t hi = n - 1u;
    while (j < hi) {
      const uint32_t mid = (j + hi) >> 1;
      if (incl[mid] > o0)
        hi = mid;
      else
        j = mid + 1u;
    }
  }
  uint32_t end_j = incl[j];
  uint32_t rec = 0, row_origin = 0, view = view0;
  int col0 = 0, width = 1, pitch = 1;
  auto load_rect = [&](uint32_t jj) {
    uint32_t cw;
    if (staged) {
      rec = s_rec[jj];
      row_origin = s_row[jj];
      cw = s_cw[jj];
      const uint32_t pv = s_pv[jj];
      pitch = (int)(pv & 0xffffu);
      view = pv >> 16;
    } else {
      const uint32_t i = g_first + jj;
      view = record_view(p, i);
      rec = p.order[i];
      row_origin = p.rect_row[i];
      cw = p.rect_cw[i];
      pitch = p.gx[view];
    }
    col0 = (int)(int16_t)(cw & 0xffffu);
    width = (int)(cw >> 16);
  };
  load_rect(j);
  // row and column of o0 in the rect: local / width from an approximate reciprocal (local < 2^21,
  // a rect holds at most every tile of a view, so the truncated estimate is within one of the
  // quotient; one step fixes it)
  const uint32_t local = o0 - (j > 0 ? incl[j - 1] : excl0);
  uint32_t ry = (uint32_t)((float)local * rcp_approx_f((float)width));
  int rem = (int)(local - ry * (uint32_t)width);
  if (rem < 0) {
    ry -= 1u;
    rem += width;
  } else if (rem >= width) {
    ry += 1u;
    rem -= width;
  }
  uint32_t keys[kEmitPerThread], vals[kEmitPerThread];
  const uint32_t slot_limit = kPerView ? (uint32_t)kSlots : 1u;
#pragma unroll
  for (int k = 0; k < kEmitPerThread; ++k) {
    const uint32_t o = o0 + (uint32_t)k;
    const bool ok = o < o_hi;
    if (k > 0 && ok) {
      // past Gaussian j: on to the next one that has instances, whose first instance o is (j stays
      // below n even after an inconsistent scan, which the status word reports)
      if (o >= end_j && j + 1u < n) {
        do {
          ++j;
          end_j = incl[j];
        } while (end_j <= o && j + 1u < n);
        load_rect(j);
        ry = 0;
        rem = 0;
      } else if (++rem == width) {
        rem = 0;
        ++ry;
      }
    }
    int tx = col0 + rem;
    if (tx < 0) tx += pitch;  // seam wrap: columns left of 0 or right of gx - 1
    if (tx >= pitch) tx -= pitch;
    const uint32_t key = row_origin + ry * (uint32_t)pitch + (uint32_t)tx;
    keys[k] = key;
    vals[k] = rec;
    // digit histograms of the tile sort (the pass that would otherwise re-read every key)
    const uint32_t slot = kPerView ? view - view0 : 0u;
    const bool counted = ok && slot < slot_limit;
    const unsigned live = __ballot_sync(kFullMask, counted);
#pragma unroll
    for (int q = 0; q < kTilePasses; ++q)
      if (q < p.hist_passes) {
        const uint32_t digit = (key >> p.hist_shift[q]) & p.hist_mask[q];
        count_digit(s_hist, slot * kHistSlot + q * kRadix + digit, counted, live, lane);
        if (kPerView && ok && !counted)
          atomicAdd(&p.hist[(size_t)view * kHistSlot + q * kRadix + digit], 1u);
      }
  }
  // the thread's run of the list: 16-byte stores when it is whole (o0 is a multiple of 8, the
  // lists start 256-byte aligned)
  static_assert(kEmitPerThread == 8, "two 16-byte stores per array");
  if (o0 + (uint32_t)kEmitPerThread <= o_hi) {
    uint4* kd = reinterpret_cast<uint4*>(p.tkeys + o0);
    uint4* vd = reinterpret_cast<uint4*>(p.tvals + o0);
    kd[0] = make_uint4(keys[0], keys[1], keys[2], keys[3]);
    kd[1] = make_uint4(keys[4], keys[5], keys[6], keys[7]);
    vd[0] = make_uint4(vals[0], vals[1], vals[2], vals[3]);
    vd[1] = make_uint4(vals[4], vals[5], vals[6], vals[7]);
  } else {
#pragma unroll
    for (int k = 0; k < kEmitPerThread; ++k)
      if (o0 + (uint32_t)k < o_hi) {
        p.tkeys[o0 + k] = keys[k];
        p.tvals[o0 + k] = vals[k];
      }
  }
  if (p.hist_passes == 0) return;
  __syncthreads();
  for (int k = threadIdx.x; k < kSlots * kHistSlot; k += kScanBlock) {
    const uint32_t c = s_hist[k];
    if (c == 0) continue;
    if (kPerView)
      atomicAdd(&p.hist[(size_t)(view0 + (uint32_t)(k / kHistSlot)) * kHistSlot + (k % kHistSlot)], c);
    else
      atomicAdd(&p.hist[k], c);
  }
}

// ---------------------------------------------------------------- tile ranges -----------------
// A thread takes kRangesPer consecutive keys (two 16-byte loads) and the key before them, so every
// load of the pass is in flight at once (one key per thread and iteration measured latency-bound:
// 25 us for the 33 MB of a 1M-Gaussian view).
constexpr int kRangesPer = 8;

__global__ void __launch_bounds__(256) ranges_kernel(RangesParams p) {
  const uint32_t L = item_count(p.hdr, 0u, p.capacity);
  const uint32_t stride = gridDim.x * blockDim.x * (uint32_t)kRangesPer;
  for (uint32_t i0 = (blockIdx.x * blockDim.x + threadIdx.x) * (uint32_t)kRangesPer; i0 < L; i0 += stride) {
    uint32_t k[kRangesPer + 1];  // k[0]: the key before i0
    k[0] = i0 > 0 ? p.keys[i0 - 1] : 0u;
    if (i0 + kRangesPer <= L) {  // i0 is a multiple of 8 and the list starts 256-byte aligned
      const uint4 a = *reinterpret_cast<const uint4*>(p.keys + i0);
      const uint4 b = *reinterpret_cast<const uint4*>(p.keys + i0 + 4);
      k[1] = a.x, k[2] = a.y, k[3] = a.z, k[4] = a.w, k[5] = b.x, k[6] = b.y, k[7] = b.z, k[8] = b.w;
    } else {
#pragma unroll
      for (int j = 0; j < kRangesPer; ++j) k[j + 1] = i0 + j < L ? p.keys[i0 + j] : 0u;
    }
#pragma unroll
    for (int j = 0; j < kRangesPer; ++j) {
      const uint32_t idx = i0 + (uint32_t)j;
      const uint32_t cur = k[j + 1], prev = k[j];
      if (idx >= L || cur >= p.num_tiles) continue;  // keys always hold valid tile ids; never index past the table
      if (idx == 0)
        p.ranges[cur].x = 0;
      else if (cur != prev) {
        if (prev < p.num_tiles) p.ranges[prev].y = idx;
        p.ranges[cur].x = idx;
      }
      if (idx == L - 1) p.ranges[cur].y = L;
    }
  }
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

void launch_histogram(const HistParams& p, int64_t max_items, cudaStream_t s) {
  const unsigned segs = p.seg_len ? std::max(1u, p.num_segs) : 1u;
  const int64_t per_seg = p.seg_len ? (int64_t)p.seg_len : max_items;
  const int64_t blocks = std::max<int64_t>(
      1, std::min<int64_t>((per_seg + 256 * kHistUnroll - 1) / (256 * kHistUnroll),
                           std::max<int64_t>(1, sm_count() * 4 / segs)));
  histogram_kernel<<<dim3((unsigned)blocks, segs), 256, 0, s>>>(p);
}

void launch_onesweep(const OnesweepParams& p, int64_t max_items, cudaStream_t s) {
  // variable segments: each segment's last tile may be partial, so up to num_segs extra tiles
  const int64_t blocks = p.seg_counts ? sort_tiles(max_items) + (int64_t)p.num_segs
                         : p.seg_len  ? sort_tiles(p.seg_len) * (int64_t)p.num_segs
                                      : sort_tiles(max_items);
  if (blocks <= 0) return;
  if (p.seg_counts)
    onesweep_kernel<true><<<(unsigned)blocks, kSortThreads, 0, s>>>(p);
  else
    onesweep_kernel<false><<<(unsigned)blocks, kSortThreads, 0, s>>>(p);
}

void launch_duplicate(const DuplicateParams& p, cudaStream_t s) {
  const int64_t items = (int64_t)p.P * p.V;
  if (items <= 0) return;
  const int64_t tiles = (items + kScanTile - 1) / kScanTile;
  if (tiles <= (int64_t)p.skip_tiles) return;
  // scan: one block per scan tile that is taken (block k takes tile skip_tiles + k)
  const unsigned blocks = (unsigned)(tiles - p.skip_tiles);
  if (p.hist_per_view)
    instance_scan_kernel<true><<<blocks, kScanBlock, 0, s>>>(p);
  else
    instance_scan_kernel<false><<<blocks, kScanBlock, 0, s>>>(p);
  // emit: one block per kEmitBlock instances the binning buffer can hold (blocks past the device's
  // instance count return at once); a probe pass stops after the scan
  if (p.skip_tiles != 0) return;
  const int64_t eblocks = emit_blocks(std::min<int64_t>(p.capacity, 0xffffffffll));
  if (eblocks <= 0) return;
  if (p.hist_per_view)
    instance_emit_kernel<true><<<(unsigned)eblocks, kScanBlock, 0, s>>>(p);
  else
    instance_emit_kernel<false><<<(unsigned)eblocks, kScanBlock, 0, s>>>(p);
}

void launch_ranges(const RangesParams& p, cudaStream_t s) {
  if (p.capacity <= 0) return;
  // enough threads for one group of keys each at the capacity (the blocks past the device count
  // return at once), at most 16 waves of 8 blocks per SM
  const int64_t per_block = 256 * kRangesPer;
  const int64_t blocks = std::max<int64_t>(
      1, std::min<int64_t>((p.capacity + per_block - 1) / per_block, (int64_t)sm_count() * 8 * 16));
  ranges_kernel<<<(unsigned)blocks, 256, 0, s>>>(p);
}

}  // namespace omnigs
