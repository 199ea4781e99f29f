// Binning: tile/depth key duplication, a stable onesweep LSD radix sort, and tile ranges.
//
// Reference: duplicateWithKeys (rasterizer_impl.cu:94-140), cub::DeviceRadixSort::SortPairs over
// key bits [0, 32 + getHigherMsb(tiles)) (:651-661), identifyTileRanges (:145-167).
//
// * duplicate: each warp owns 32 consecutive Gaussians, whose instances occupy one contiguous
//   output span (their offsets are consecutive).  The warp walks that span 32 instances at a time,
//   finds each instance's owner with a 5-step shuffle search over the lanes' start offsets, and
//   writes keys/values fully coalesced, so a splat covering hundreds of tiles no longer serialises
//   one thread.  The same pass accumulates the 8-bit digit histograms of every sort pass.
// * sort: one kernel per 8-bit digit.  A block ranks a 4096-key tile in shared memory (warp
//   multi-split with match.any, which keeps equal digits in input order, so the sort is stable),
//   publishes its per-digit counts, resolves its global digit offsets by decoupled look-back
//   (blocks take tiles in launch order from an atomic counter) and scatters.  A stable LSD sort
//   over the same bit range yields exactly cub's order: by key, ties in unsorted order.
// * ranges: per-tile [start, end) over the sorted keys.
// Instance counts live only on the device; every kernel reads num_rendered from the geometry
// header and does nothing if it exceeds the binning capacity.
#include <algorithm>

#include "device_util.cuh"
#include "kernels.h"
#include "lonlat_math.cuh"

namespace omnigs {
namespace {

constexpr uint32_t kLbAggregate = 1u << 30;
constexpr uint32_t kLbPrefix = 2u << 30;
constexpr uint32_t kLbValue = (1u << 30) - 1;
constexpr int kDupThreads = 256;
constexpr int kLookbackBatch = 8;

__device__ __forceinline__ bool capacity_ok(const GeomHeader* hdr, int64_t capacity) {
  const unsigned long long R = hdr->num_rendered64;
  return (hdr->status & kStatusOverflow) == 0 && R <= (unsigned long long)capacity;
}

__global__ void __launch_bounds__(kDupThreads) duplicate_kernel(DuplicateParams p) {
  __shared__ uint32_t s_hist[kMaxSortPasses][kRadix];
  for (int i = threadIdx.x; i < kMaxSortPasses * kRadix; i += kDupThreads) (&s_hist[0][0])[i] = 0;
  __syncthreads();
  if (!capacity_ok(p.hdr, p.capacity)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&p.hdr->status, kStatusCapacity);
    return;
  }
  const uint32_t R = p.hdr->num_rendered;
  // clear the sort look-back words of the tiles this sort will use
  {
    const int64_t ntiles = (R + kSortTile - 1) / kSortTile;
    const int64_t n = ntiles * kRadix;
    for (int pass = 0; pass < p.passes; ++pass)
      for (int64_t i = blockIdx.x * (int64_t)kDupThreads + threadIdx.x; i < n;
           i += (int64_t)gridDim.x * kDupThreads)
        p.lookback[pass * p.lookback_pass_stride + i] = 0;
  }
  const int lane = threadIdx.x & 31;
  const int warps_total = gridDim.x * (kDupThreads / 32);
  for (int base = (blockIdx.x * (kDupThreads / 32) + (threadIdx.x >> 5)) * 32; base < p.P;
       base += warps_total * 32) {
    const int g = base + lane;
    uint32_t start = R, count = 0, dbits = 0;
    int rminx = 0, rminy = 0, width = 1;
    if (g < p.P) {
      start = (g == 0) ? 0u : p.offsets[g - 1];
      const int radius = p.radii[g];
      if (radius > 0) {
        const float4 a = p.splat[2 * g];
        int2 rmin, rmax;
        tile_rect(make_float2(a.x, a.y), radius, p.gx, p.gy, rmin, rmax);
        rminx = rmin.x;
        rminy = rmin.y;
        width = rmax.x - rmin.x;
        count = p.offsets[g] - start;
        dbits = __float_as_uint(p.depth[g]);
      }
    }
    const uint32_t w_begin = __shfl_sync(kFullMask, start, 0);
    const uint32_t w_end = __shfl_sync(kFullMask, start + count, 31);
    for (uint32_t o0 = w_begin; o0 < w_end; o0 += 32) {
      const uint32_t o = o0 + lane;
      const bool valid = o < w_end;
      int pos = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t s = __shfl_sync(kFullMask, start, pos + step);
        if (s <= o) pos += step;
      }
      const uint32_t o_start = __shfl_sync(kFullMask, start, pos);
      const int o_rminx = __shfl_sync(kFullMask, rminx, pos);
      const int o_rminy = __shfl_sync(kFullMask, rminy, pos);
      const int o_width = __shfl_sync(kFullMask, width, pos);
      const uint32_t o_dbits = __shfl_sync(kFullMask, dbits, pos);
      uint64_t key = 0;
      if (valid) {
        const uint32_t local = o - o_start;
        const uint32_t ty = (uint32_t)o_rminy + local / (uint32_t)o_width;
        const uint32_t tx = (uint32_t)o_rminx + local % (uint32_t)o_width;
        key = ((uint64_t)(ty * (uint32_t)p.gx + tx) << 32) | o_dbits;
        p.keys[o] = key;
        p.vals[o] = (uint32_t)(base + pos);
      }
      for (int pass = 0; pass < p.passes; ++pass) {
        const uint32_t digit = (uint32_t)(key >> (kRadixBits * pass)) & (kRadix - 1);
        const uint32_t tag = valid ? digit : (0x10000u + lane);
        const unsigned peers = __match_any_sync(kFullMask, tag);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&s_hist[pass][digit], (uint32_t)__popc(peers));
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < p.passes * kRadix; i += kDupThreads) {
    const uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(&p.hist[i], v);
  }
}

// Dynamic shared memory of one sort tile.
struct SortSmem {
  uint32_t warp_hist[kSortThreads / 32][kRadix];
  uint32_t block_excl[kRadix];
  uint32_t global_base[kRadix];
  uint32_t scan_tmp[kSortThreads / 32];
  uint32_t tile;
  uint32_t pad[3];
  uint64_t keys[kSortTile];
  uint32_t vals[kSortTile];
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

__global__ void __launch_bounds__(kSortThreads) sort_pass_kernel(SortPassParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SortSmem& sm = *reinterpret_cast<SortSmem*>(smem_raw);
  if (!capacity_ok(p.hdr, p.capacity)) return;
  const uint32_t R = p.hdr->num_rendered;
  const uint32_t ntiles = (R + kSortTile - 1) / kSortTile;
  if (threadIdx.x == 0) sm.tile = atomicAdd(p.tile_counter, 1u);
  for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&sm.warp_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = sm.tile;
  if (tile >= ntiles) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;

  // where each digit starts in the whole output
  uint32_t unused;
  sm.global_base[threadIdx.x] = block_exclusive_scan(p.hist[threadIdx.x], sm.scan_tmp, unused);

  // load (warp-striped) and rank within the warp; match.any groups equal digits and the lanes
  // of a group are ranked in lane order, items in k order: a stable multi-split.
  uint64_t key[kSortItems];
  uint32_t val[kSortItems];
  uint32_t rank[kSortItems];
  const uint32_t tile_base = tile * kSortTile + warp * (kSortItems * 32);
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t idx = tile_base + k * 32 + lane;
    const bool valid = idx < R;
    key[k] = valid ? p.keys_in[idx] : 0ull;
    val[k] = valid ? p.vals_in[idx] : 0u;
    const uint32_t digit = (uint32_t)(key[k] >> p.shift) & (kRadix - 1);
    const unsigned peers = __match_any_sync(kFullMask, valid ? digit : (0x10000u + lane));
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (valid && lane == leader) {
      old = sm.warp_hist[warp][digit];
      sm.warp_hist[warp][digit] = old + __popc(peers);
    }
    old = __shfl_sync(kFullMask, old, leader);
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

  // decoupled look-back for this digit
  uint32_t* lb = p.lookback;
  if (tile == 0) {
    st_relaxed_u32(&lb[d], kLbPrefix | count);
  } else {
    st_relaxed_u32(&lb[(size_t)tile * kRadix + d], kLbAggregate | count);
    uint32_t prev = 0;
    int64_t j = (int64_t)tile - 1;
    bool gave_up = false;
    bool found = false;
    while (!found) {
      uint32_t w[kLookbackBatch];
#pragma unroll
      for (int b = 0; b < kLookbackBatch; ++b)
        w[b] = (j - b >= 0) ? ld_relaxed_u32(&lb[(size_t)(j - b) * kRadix + d]) : kLbPrefix;
#pragma unroll
      for (int b = 0; b < kLookbackBatch; ++b) {
        if (found) break;
        uint32_t x = w[b];
        if ((x >> 30) == 0) {
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
        prev += x & kLbValue;
        if ((x >> 30) == 2) found = true;
      }
      j -= kLookbackBatch;
    }
    if (gave_up) atomicOr(&p.hdr->status, kStatusLookback);
    st_relaxed_u32(&lb[(size_t)tile * kRadix + d], kLbPrefix | ((prev + count) & kLbValue));
    sm.global_base[d] += prev;
  }

  // scatter into shared memory in digit order
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    if (rank[k] != 0xffffffffu) {
      const uint32_t digit = (uint32_t)(key[k] >> p.shift) & (kRadix - 1);
      const uint32_t pos = sm.block_excl[digit] + sm.warp_hist[warp][digit] + rank[k];
      if (pos < (uint32_t)kSortTile) {  // always true: ranks are consistent within the block
        sm.keys[pos] = key[k];
        sm.vals[pos] = val[k];
      }
    }
  }
  __syncthreads();
  // write runs of equal digits to their global positions
  for (uint32_t i = threadIdx.x; i < tile_items; i += kSortThreads) {
    const uint64_t k64 = sm.keys[i];
    const uint32_t digit = (uint32_t)(k64 >> p.shift) & (kRadix - 1);
    const uint32_t out = sm.global_base[digit] + (i - sm.block_excl[digit]);
    if (out < R) {  // always true unless a look-back gave up (then the status word says so)
      p.keys_out[out] = k64;
      p.vals_out[out] = sm.vals[i];
    }
  }
}

__global__ void ranges_kernel(RangesParams p) {
  if (!capacity_ok(p.hdr, p.capacity)) return;
  const uint32_t L = p.hdr->num_rendered;
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= L) return;
  const uint32_t cur = (uint32_t)(p.keys[idx] >> 32);
  if (cur >= p.num_tiles) return;  // keys always hold valid tile ids; never index past the table
  if (idx == 0)
    p.ranges[cur].x = 0;
  else {
    const uint32_t prev = (uint32_t)(p.keys[idx - 1] >> 32);
    if (cur != prev) {
      if (prev < p.num_tiles) p.ranges[prev].y = idx;
      p.ranges[cur].x = idx;
    }
  }
  if (idx == L - 1) p.ranges[cur].y = L;
}

}  // namespace

void launch_duplicate(const DuplicateParams& p, cudaStream_t s) {
  if (p.P <= 0) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int warps_needed = (p.P + 31) / 32;
  const int blocks = std::max(1, std::min((warps_needed + 7) / 8, sms * 8));
  duplicate_kernel<<<blocks, kDupThreads, 0, s>>>(p);
}

void launch_sort_pass(const SortPassParams& p, cudaStream_t s) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    cudaFuncSetAttribute(sort_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SortSmem));
    if (dev >= 0 && dev < 64) configured[dev] = true;
  }
  const int64_t blocks = BinningLayout::sort_tiles(p.capacity);
  if (blocks <= 0) return;
  sort_pass_kernel<<<(unsigned)blocks, kSortThreads, sizeof(SortSmem), s>>>(p);
}

void launch_ranges(const RangesParams& p, cudaStream_t s) {
  if (p.capacity <= 0) return;
  const int64_t blocks = (p.capacity + 255) / 256;
  ranges_kernel<<<(unsigned)blocks, 256, 0, s>>>(p);
}

}  // namespace omnigs
