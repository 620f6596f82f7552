// Stable LSD radix sort of uint32 keys with uint32 values for sm_100a: a
// counting kernel reads the keys once (every digit place's histogram, valid
// keys per tile and per segment), then one onesweep kernel per 8-bit digit
// place. Each onesweep tile ranks its keys with a warp multisplit (one ballot
// per digit bit) in shared memory, publishes its digit counts and finds its
// global offsets by decoupled lookback (single pass, no separate scan
// kernel), then scatters keys and values through shared memory so writes of
// one digit run are contiguous. Kernels after the first start by programmatic
// dependent launch.
//
// The largest key of a width (2^bits - 1, the invalid key of SortKeys) sorts
// after every other key, its copies in input order. When outputs do not alias
// inputs, a stable partition kernel (offsets from per-tile valid counts that
// the counting kernel wrote, no digit ranking) first writes them straight to the tail
// of each segment's output and packs the other keys, in order, at the
// segment's front; every digit pass then sorts only those: a frame's culled
// splats are read twice and written once, never ranked.
//
// Replaces WgpuRadixSort (src/wgpu/WgpuRadixSort.ts:43-361: 3 dispatches per
// pass, histogram / scanBlocks / scatter with 8 one-bit splits), WgpuCompact
// + sortIndirect as the splat sorter uses them, and SortKeys.sort
// (src/core/sort.ts:64-163). Any stable ascending sort yields their order.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "rdx_internal.h"

namespace rdx {
namespace {

// Lookback word: epoch (32) | flag (2) | count (30)
constexpr uint64_t kFlagAggregate = 1ull << 30;
constexpr uint64_t kFlagInclusive = 2ull << 30;
constexpr uint64_t kFlagMask = 3ull << 30;
constexpr uint64_t kCountMask = (1ull << 30) - 1ull;
constexpr uint32_t kNotRanked = 0xffffu;  // the digit of an item outside the ranking
constexpr int kSortBlocksPerSm = 4;       // onesweep blocks resident per SM (register budget)
constexpr int kCountBlocksPerSm = 8;      // counting blocks resident per SM (one wave at 4M keys)

__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Lanes whose item has the same digit as this lane's (ranked items only; the
// unranked ones group among themselves): one ballot per digit bit, cheaper
// than a general match over 32-bit values
__device__ __forceinline__ uint32_t peers_of(uint32_t d, bool ranked) {
  const uint32_t r = __ballot_sync(0xffffffffu, ranked);
  uint32_t peers = ranked ? r : ~r;
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const bool bit = (d >> b) & 1u;
    const uint32_t m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

// The same over the low `nbits` bits of a code that is unique per digit present
// (a place holding few distinct digits ranks with fewer ballots); nbits is
// uniform over the block
__device__ __forceinline__ uint32_t peers_of_code(uint32_t c, bool ranked, int nbits) {
  const uint32_t r = __ballot_sync(0xffffffffu, ranked);
  uint32_t peers = ranked ? r : ~r;
#pragma unroll
  for (int b = 0; b < 8; b++) {
    if (b < nbits) {
      const bool bit = (c >> b) & 1u;
      const uint32_t m = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? m : ~m;
    }
  }
  return peers;
}

// Segment holding `tile` (seg_tiles is non-decreasing, seg_tiles[0] = 0)
__device__ __forceinline__ int segment_of(const uint32_t* seg_tiles, int count, uint32_t tile) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg_tiles[mid] <= tile) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

// Exclusive scan over the 256 threads of a block (64-bit lanes); `sums` is
// 8 words of shared memory. Returns the thread's exclusive prefix; *total the sum.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* sums, uint64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint64_t s = lane < kSortWarps ? sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < kSortWarps; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kSortWarps) sums[lane] = s;  // inclusive warp totals
  }
  __syncthreads();
  *total = sums[kSortWarps - 1];
  const uint64_t before = warp > 0 ? sums[warp - 1] : 0;
  return before + x - v;
}

// ---- counting: every digit place's histogram, valid keys per tile and segment ----

// One block per tile: the tile's keys in one read give every digit place's
// histogram of the valid keys (one 32-bit shared-memory histogram a place for
// the block, one shared atomic per key and place: the hardware merges the
// lanes of a warp that add to one bin; summed into the segment's by one global
// atomic per non-zero bin), the tile's valid count
// (the partition's offsets), the segment's valid count and the reference's
// hidden count. Block 0 also advances the lookback epoch: the word is bumped
// on the device, so a sort replayed from a CUDA graph still tags its words
// with a new epoch.
// TOP_ONLY: only the top place's histogram (what the cooperative digit passes
// need; they sum the other places' digit totals from their blocks' counts)
template <int PASSES, bool TOP_ONLY>
__global__ void __launch_bounds__(kSortThreads, kCountBlocksPerSm)
    k_sort_count(const uint32_t* __restrict__ keys, uint32_t key_mask, int ref_shift, uint32_t ref_top, int drop,
                 SortSegments segs, uint32_t* __restrict__ hist, uint32_t* __restrict__ valid_count,
                 uint32_t* __restrict__ ref_hidden, uint32_t* __restrict__ tile_valid, uint32_t* epoch) {
  static_assert(kSortThreads == kRadix, "a thread a bin");
  constexpr int kFirst = TOP_ONLY ? PASSES - 1 : 0;  // the first place counted
  __shared__ uint32_t sh[PASSES - kFirst][kRadix];
  __shared__ uint32_t s_valid[kSortWarps], s_hidden[kSortWarps];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
#pragma unroll
  for (int p = 0; p < PASSES - kFirst; p++) sh[p][tid] = 0;
  __syncthreads();
  pdl_wait();
  pdl_trigger();
  if (tid == 0 && blockIdx.x == 0) {
    const uint32_t e = *epoch + 1u;
    *epoch = e == 0u ? 1u : e;  // 0 marks a cleared word
  }
  const uint32_t tile = blockIdx.x;
  if (tile >= segs.tiles[segs.count]) return;  // grid sized for the capacity
  const int seg = segment_of(segs.tiles, segs.count, tile);
  const uint64_t base = segs.begin[seg] + (uint64_t)(tile - segs.tiles[seg]) * kSortTile;
  const uint32_t n = (uint32_t)min((uint64_t)kSortTile, segs.end[seg] - base);
  const uint32_t warp_base = (uint32_t)warp * (kSortItems * 32);
  uint32_t key[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    key[j] = pos < n ? __ldg(&keys[base + pos]) & key_mask : key_mask;
  }
  __syncwarp();
  uint32_t nvalid = 0, hidden = 0;
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    const bool in = pos < n;
    hidden += in && (key[j] >> ref_shift) == ref_top;
    const bool valid = in && (!drop || key[j] != key_mask);
    nvalid += valid;
    if (valid) {
#pragma unroll
      for (int p = kFirst; p < PASSES; p++) atomicAdd(&sh[p - kFirst][(key[j] >> (8 * p)) & 0xffu], 1u);
    }
  }
  nvalid = __reduce_add_sync(0xffffffffu, nvalid);
  hidden = __reduce_add_sync(0xffffffffu, hidden);
  if (lane == 0) {
    s_valid[warp] = nvalid;
    s_hidden[warp] = hidden;
  }
  __syncthreads();
  // thread d adds bin d of every place to the segment's histogram
  const uint32_t d = (uint32_t)tid;
#pragma unroll
  for (int p = kFirst; p < PASSES; p++) {
    const uint32_t c = sh[p - kFirst][d];
    if (c) atomicAdd(&hist[((size_t)seg * PASSES + p) * kRadix + d], c);
  }
  if (tid == 0) {
    uint32_t v = 0, h = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
      v += s_valid[w];
      h += s_hidden[w];
    }
    tile_valid[tile] = v;
    if (v) atomicAdd(&valid_count[seg], v);
    if (h) atomicAdd(&ref_hidden[seg], h);
  }
}

// ---- stable partition: the valid keys packed at each segment's front ----

struct PartArgs {
  const uint32_t* keys_in;
  const uint32_t* vals_in;  // null: each key's index within its segment
  uint32_t* keys_front;     // valid keys at begin[s] + their rank among the segment's valid keys
  uint32_t* vals_front;
  uint32_t* tail_keys;      // largest keys (final outputs; may be null) at begin[s] + valid[s] + rank
  uint32_t* tail_vals;
  uint32_t key_mask;
  SortSegments segs;
  const uint32_t* valid_count;
  const uint32_t* tile_valid;  // [tiles] valid keys of each tile, complete before this kernel
  uint32_t* counter;
  uint64_t* vbegin;            // out (block 0): the valid keys' segments for the digit passes
  uint64_t* vend;
  uint32_t* vtiles;            // in tiles of pass_tile keys
  uint32_t pass_tile;
  uint32_t* error_flag;
  uint32_t* visible;           // out (block 0, may be null): each segment's visible count
  const uint32_t* ref_hidden;  // the reference's count of it (null: the valid keys)
};

constexpr int kPartBlocksPerSm = 8;

// Each tile's offsets come from the valid counts of the segment's earlier
// tiles, which the counting kernel wrote: no tile waits for another.
__global__ void __launch_bounds__(kSortThreads, kPartBlocksPerSm) k_partition(PartArgs a) {
  __shared__ uint32_t s_warp_valid[kSortWarps];
  __shared__ uint32_t s_warp_prefix[kSortWarps];
  __shared__ uint32_t s_tile;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  pdl_wait();
  pdl_trigger();
  if (tid == 0 && blockIdx.x == 0) {
    // The valid keys' segments [begin, begin + valid) and their tiles; the visible counts
    uint32_t t = 0;
    for (int s = 0; s < a.segs.count; s++) {
      const uint64_t b = a.segs.begin[s];
      const uint64_t v = min((uint64_t)a.valid_count[s], a.segs.end[s] - b);
      a.vbegin[s] = b;
      a.vend[s] = b + v;
      a.vtiles[s] = t;
      t += (uint32_t)((v + a.pass_tile - 1) / a.pass_tile);
      if (a.visible) a.visible[s] = a.ref_hidden ? (uint32_t)(a.segs.end[s] - b) - a.ref_hidden[s] : a.valid_count[s];
    }
    a.vtiles[a.segs.count] = t;
  }
  if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  if (tile >= a.segs.tiles[a.segs.count]) return;
  const int seg = segment_of(a.segs.tiles, a.segs.count, tile);
  const uint32_t first = a.segs.tiles[seg];
  const uint32_t local_tile = tile - first;
  const uint64_t seg_begin = a.segs.begin[seg];
  const uint64_t seg_end = a.segs.end[seg];
  const uint64_t base = seg_begin + (uint64_t)local_tile * kSortTile;
  const uint32_t n = (uint32_t)min((uint64_t)kSortTile, seg_end - base);
  const uint32_t warp_base = (uint32_t)warp * (kSortItems * 32);
  const uint32_t lt = lanemask_lt();

  // Warp w holds tile positions [w * 512, (w + 1) * 512), item j at j * 32 + lane
  uint32_t key[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    key[j] = pos < n ? __ldg(&a.keys_in[base + pos]) & a.key_mask : a.key_mask;
  }
  // Valid keys of the segment's earlier tiles (loads in flight with the keys')
  uint32_t before = 0;
#pragma unroll 4
  for (uint32_t t = first + (uint32_t)tid; t < tile; t += kSortThreads) before += __ldg(&a.tile_valid[t]);
  uint32_t warp_valid = 0;
#pragma unroll
  for (int j = 0; j < kSortItems; j++) warp_valid += (uint32_t)__popc(__ballot_sync(0xffffffffu, key[j] != a.key_mask));
  before = __reduce_add_sync(0xffffffffu, before);
  if (lane == 0) {
    s_warp_valid[warp] = warp_valid;
    s_warp_prefix[warp] = before;
  }
  __syncthreads();
  uint32_t valid_before = 0, warp_before = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    warp_before += w < warp ? s_warp_valid[w] : 0u;
    valid_before += s_warp_prefix[w];
  }

  // Valid keys to the front in order; the largest keys to the tail in order
  const uint32_t seg_valid = min(a.valid_count[seg], (uint32_t)(seg_end - seg_begin));
  const uint64_t front = seg_begin + valid_before;
  const uint64_t tail = seg_begin + seg_valid + ((uint64_t)local_tile * kSortTile - valid_before);
  uint32_t run = warp_before;
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    const bool valid = key[j] != a.key_mask;
    const uint32_t vb = __ballot_sync(0xffffffffu, valid);
    const uint32_t r = run + (uint32_t)__popc(vb & lt);  // valid keys of the tile before this one
    run += (uint32_t)__popc(vb);
    if (pos < n) {
      const uint32_t value = a.vals_in ? __ldg(&a.vals_in[base + pos]) : (uint32_t)(base - seg_begin) + pos;
      if (valid) {
        const uint64_t dst = front + r;
        if (dst < seg_begin + seg_valid) {
          a.keys_front[dst] = key[j];
          a.vals_front[dst] = value;
        } else {
          check_failed(a.error_flag);
        }
      } else {
        const uint64_t dst = tail + (pos - r);
        if (dst < seg_end) {
          a.tail_vals[dst] = value;
          if (a.tail_keys) a.tail_keys[dst] = key[j];
        } else {
          check_failed(a.error_flag);
        }
      }
    }
  }
}

// ---- onesweep: one digit place ----

struct PassArgs {
  const uint32_t* keys_in;
  const uint32_t* vals_in;   // null (first pass of an in-place sort): each key's index within its segment
  uint32_t* keys_out;        // null: values only
  uint32_t* vals_out;
  uint32_t key_mask;
  int shift;
  SortSegments segs;         // the valid keys' segments (after a partition) or the segments as given
  const uint32_t* hist;      // [S][passes][256] of the keys sorted
  int passes;
  int place;
  uint64_t* lookback;        // [max_tiles][256] of this pass
  const uint32_t* epoch;     // this sort's lookback epoch (device word)
  uint32_t* counter;
  uint32_t* error_flag;
  uint32_t spin_limit;       // polls of a lookback word before a tile gives up
  uint32_t silent_tile;      // a tile that publishes no lookback word (a test of the bounded wait; ~0u: none)
};

template <bool FIRST, bool WRITE_KEYS, int ITEMS>
__global__ void __launch_bounds__(kSortThreads, kSortBlocksPerSm) k_onesweep(PassArgs a) {
  constexpr int TILE = kSortThreads * ITEMS;
  __shared__ uint32_t s_whist[kSortWarps][kRadix];
  __shared__ uint32_t s_exchange[TILE];
  __shared__ uint32_t s_vals[TILE];  // the tile's values, copied in asynchronously
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_dest[kRadix];
  __shared__ uint64_t s_sums[kSortWarps];
  __shared__ uint32_t s_tile;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

#pragma unroll
  for (int w = 0; w < kSortWarps; w++) s_whist[w][tid] = 0;
  pdl_wait();     // the previous pass (or the set-up) has completed
  pdl_trigger();  // the next pass may start placing its blocks
  if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t total_tiles = a.segs.tiles[a.segs.count];
  if (tile >= total_tiles) return;  // grid sized for the capacity

  const int seg = segment_of(a.segs.tiles, a.segs.count, tile);
  const uint32_t local_tile = tile - a.segs.tiles[seg];
  const uint64_t seg_begin = a.segs.begin[seg];
  const uint64_t seg_end = a.segs.end[seg];
  const uint64_t base = seg_begin + (uint64_t)local_tile * TILE;
  const uint32_t n = (uint32_t)min((uint64_t)TILE, seg_end - base);

  // Load: warp w holds tile positions [w * 512, (w + 1) * 512), item j at j * 32 + lane.
  // Keys go to registers; values go straight to shared memory (cp.async, no
  // registers held) and are waited for only before they are scattered. In the
  // first pass without values, a value is the key's index within its segment.
  const bool gen_vals = FIRST && a.vals_in == nullptr;
  uint32_t key[ITEMS], rank[ITEMS];
  const uint32_t warp_base = (uint32_t)warp * (ITEMS * 32);
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    if (pos < n) {
      key[j] = __ldg(&a.keys_in[base + pos]) & a.key_mask;
      if (!gen_vals) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_vals[pos])),
                     "l"(&a.vals_in[base + pos])
                     : "memory");
      }
    } else {
      key[j] = 0u;
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  auto value_at = [&](uint32_t pos) -> uint32_t {
    return gen_vals ? (uint32_t)(base - seg_begin) + pos : s_vals[pos];
  };

  // Rank the keys: items in position order, equal digits counted by their lowest lane
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    const bool ranked = pos < n;
    const uint32_t d = ranked ? (key[j] >> a.shift) & 0xffu : kNotRanked;
    const uint32_t peers = peers_of(d, ranked);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (lane == leader && d != kNotRanked) {
      old = s_whist[warp][d];
      s_whist[warp][d] = old + (uint32_t)__popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[j] = old + (uint32_t)__popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();

  // Thread d owns digit d: warp counts -> exclusive over warps, the tile's count
  const uint32_t d = (uint32_t)tid;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = s_whist[w][d];
    s_whist[w][d] = total;
    total += c;
  }
  uint64_t* my_word = &a.lookback[(size_t)tile * kRadix + d];
  const uint32_t epoch = *a.epoch;
  const uint64_t ep = (uint64_t)epoch << 32;
  const bool silent = tile == a.silent_tile;
  if (!silent) st_relaxed64(my_word, ep | (local_tile == 0 ? kFlagInclusive : kFlagAggregate) | total);

  // Tile-local digit starts (low word) and the segment's digit offsets (high word) in one scan
  const uint32_t seg_count = a.hist[((size_t)seg * a.passes + a.place) * kRadix + d];
  uint64_t both_total;
  const uint64_t both = block_exclusive_scan(((uint64_t)seg_count << 32) | total, s_sums, &both_total);
  const uint32_t tile_start = (uint32_t)both;
  const uint32_t tile_count = (uint32_t)both_total;
  const uint32_t seg_digit = (uint32_t)(both >> 32);
  s_tile_start[d] = tile_start;

  // Decoupled lookback over this segment's earlier tiles, bounded
  uint32_t prefix = 0;
  if (local_tile > 0) {
    uint32_t t = tile - 1;
    uint32_t spins = 0;
    while (true) {
      const uint64_t v = ld_relaxed64(&a.lookback[(size_t)t * kRadix + d]);
      const uint64_t flag = (v >> 32) == epoch ? (v & kFlagMask) : 0;
      if (flag == 0) {
        if (++spins > a.spin_limit) {
          atomicOr(a.error_flag, kErrTimeout);
          break;
        }
        if (spins > 32) __nanosleep(32);
        continue;
      }
      prefix += (uint32_t)(v & kCountMask);
      if (flag == kFlagInclusive) break;
      t--;
    }
    if (!silent) st_relaxed64(my_word, ep | kFlagInclusive | (prefix + total));
  }
  s_dest[d] = (uint32_t)seg_begin + seg_digit + prefix - tile_start;
  asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's value copies have landed
  __syncthreads();                                   // and every thread's

  // Local sort of the tile's keys in shared memory
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    if (pos < n) {
      const uint32_t dj = (key[j] >> a.shift) & 0xffu;
      rank[j] += s_tile_start[dj] + s_whist[warp][dj];
      s_exchange[rank[j]] = key[j];
    } else {
      rank[j] = 0xffffffffu;
    }
  }
  __syncthreads();
  // Destinations stay inside the segment even if a bounded wait gave up
  uint32_t dest[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; k++) {
    const uint32_t i = (uint32_t)k * kSortThreads + tid;
    dest[k] = 0xffffffffu;
    if (i < tile_count) {
      const uint32_t kk = s_exchange[i];
      const uint32_t dst = s_dest[(kk >> a.shift) & 0xffu] + i;
      if (dst >= (uint32_t)seg_begin && dst < (uint32_t)seg_end) {
        dest[k] = dst;
        if (WRITE_KEYS) a.keys_out[dst] = kk;
      } else {
        check_failed(a.error_flag);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; j++) {
    if (rank[j] != 0xffffffffu) s_exchange[rank[j]] = value_at(warp_base + (uint32_t)j * 32 + lane);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; k++) {
    const uint32_t i = (uint32_t)k * kSortThreads + tid;
    if (dest[k] != 0xffffffffu) a.vals_out[dest[k]] = s_exchange[i];
  }
}

// ---- cooperative: every digit pass of one segment in one persistent kernel ----
//
// One block per SM slot, all resident (a cooperative launch). Block b owns
// the keys [b * C, (b + 1) * C) of each pass's input (C = V / blocks, a
// multiple of 4), in sub-tiles of THREADS * ITEMS keys. A pass: the block
// ranks its keys (the same warp multisplit as the onesweep) and publishes its
// 256 digit counts; after a grid barrier every block sums the earlier blocks'
// counts per digit (its offsets, no chain of predecessors to wait on) and
// scatters through shared memory; a second barrier ends the pass. When a
// block's keys fit one sub-tile they stay in registers across the barrier.
// Data written by other blocks of this kernel is read through L2 only (.cg):
// an SM's L1 may still hold lines of the same buffer from two passes before.

struct CoopArgs {
  const uint32_t* keys_in;   // the first pass's input
  const uint32_t* vals_in;   // null: each key's index within the segment
  uint32_t* keys_a;          // ping-pong pairs
  uint32_t* vals_a;
  uint32_t* keys_b;
  uint32_t* vals_b;
  uint32_t* keys_out;        // the last pass's keys (null: values only)
  uint32_t* vals_out;
  const uint64_t* begin;     // the segment sorted: [begin[0], end[0])
  const uint64_t* end;
  const uint32_t* hist;      // [passes][256]: the top place's digit counts of the keys sorted
  uint32_t* block_counts;    // [blocks][256]
  uint32_t* barrier;         // grid-barrier arrivals of this sort (zero at its start)
  uint32_t* error_flag;
  uint32_t key_mask;
  int passes;
  int drop;                  // the first pass reads the partition's A buffers (ping-pong B, A, ...)
  uint32_t spin_limit;
  int silent_pass;           // test hook: block 0 does not arrive at that pass's first barrier
};

__device__ __forceinline__ uint32_t ld_acquire32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier (every block resident): the sort's `count`-th. A wait is
// bounded: after spin_limit polls the block sets the error flag and goes on.
__device__ __forceinline__ void grid_barrier(const CoopArgs& a, uint32_t target, bool arrive) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (arrive) atomicAdd(a.barrier, 1u);
    uint32_t spins = 0;
    while (ld_acquire32(a.barrier) < target) {
      if (++spins > a.spin_limit) {
        atomicOr(a.error_flag, kErrTimeout);
        break;
      }
      if (spins > 16) __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
}

// Exclusive scan of one value per digit (threads 0-255; the others pass 0 and
// get 0) over a block of THREADS; warp_sums: 8 words of shared memory
template <int THREADS>
__device__ __forceinline__ uint32_t digit_exclusive_scan(uint32_t v, uint32_t* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (warp < kRadix / 32 && lane == 31) warp_sums[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  if (warp < kRadix / 32) {
#pragma unroll
    for (int w = 0; w < kRadix / 32; w++) before += w < warp ? warp_sums[w] : 0u;
  }
  __syncthreads();
  return warp < kRadix / 32 ? before + x - v : 0u;
}

template <int THREADS, int ITEMS>
struct CoopShape {
  static constexpr int kWarps = THREADS / 32;
  static constexpr uint32_t kSub = THREADS * ITEMS;  // keys of a sub-tile
  // shared words: per-warp digit counts, exchange, values, and 256-word tables
  static constexpr size_t kWords = (size_t)kWarps * kRadix + 2 * (size_t)kSub + (8 + kMaxPasses) * kRadix + 32;
  static constexpr size_t kBytes = kWords * 4;
};

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_sort_coop(CoopArgs a) {
  using Shape = CoopShape<THREADS, ITEMS>;
  constexpr int kWarps = Shape::kWarps;
  constexpr uint32_t kSub = Shape::kSub;
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_whist = smem;                            // [warps][256]: counts, then exclusive over warps
  uint32_t* s_exchange = s_whist + kWarps * kRadix;    // [kSub]
  uint32_t* s_vals = s_exchange + kSub;                // [kSub]: the sub-tile's values (cp.async)
  uint32_t* s_cnt = s_vals + kSub;                     // [256] the sub-tile's digit counts
  uint32_t* s_start = s_cnt + kRadix;                  // [256] their exclusive scan (tile-local starts)
  uint32_t* s_blk = s_start + kRadix;                  // [256] the block's digit counts of this pass
  uint32_t* s_base = s_blk + kRadix;                   // [256] the next destination of each digit
  uint32_t* s_part = s_base + kRadix;                  // [4][256] partial sums (earlier blocks, warp groups)
  uint32_t* s_code = s_part + 4 * kRadix;              // [passes][256] each present digit's compact code
  uint32_t* s_wsum = s_code + kMaxPasses * kRadix;     // [8] scan scratch, [9 + place]: the place's code bits

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const uint32_t G = gridDim.x;
  const uint32_t b = blockIdx.x;
  const uint64_t seg_begin = a.begin[0];
  const uint32_t V = (uint32_t)min(a.end[0] - seg_begin, (uint64_t)kMaxSegmentKeys);
  const uint32_t C = (((V + G - 1) / G) + 3u) & ~3u;
  const uint32_t lo = min(b * C, V);
  const uint32_t len = min(C, V - lo);
  const uint32_t nsub = (len + kSub - 1) / kSub;
  const uint32_t warp_base = (uint32_t)warp * (ITEMS * 32);
  const uint32_t lt = lanemask_lt();
  uint32_t key[ITEMS], rank[ITEMS];
  uint32_t barriers = 0;
  const uint32_t* kin = a.keys_in;
  const uint32_t* vin = a.vals_in;

  // Load sub-tile `sub` (keys to registers, values to s_vals when `vals`) and
  // rank it: rank[j] = earlier items of its digit in the warp, s_cnt = the
  // sub-tile's counts, s_start their exclusive scan, s_whist exclusive over warps
  auto load_rank = [&](uint32_t sub, int shift, bool vals) -> uint32_t {
    const uint64_t start = seg_begin + lo + (uint64_t)sub * kSub;
    const uint32_t n = min(kSub, len - sub * kSub);
    for (int w = tid; w < kWarps * kRadix; w += THREADS) s_whist[w] = 0;
    if (vals && vin) {
      // whole 16-byte groups of values straight to shared memory (L2 only); the tail at use
      const bool vec = (reinterpret_cast<uintptr_t>(vin + start) & 15u) == 0;
      const uint32_t groups = vec ? n / 4 : 0;
      for (uint32_t g = tid; g < groups; g += THREADS) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_vals[4 * g])),
                     "l"(vin + start + 4 * g)
                     : "memory");
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
      const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
      key[j] = pos < n ? __ldcg(&kin[start + pos]) & a.key_mask : 0u;
    }
    __syncthreads();  // s_whist cleared
    if (warp_base < n) {  // warps past the sub-tile's keys have nothing to rank
      const int nbits = (int)s_wsum[9 + shift / 8];
      uint32_t* h = s_whist + warp * kRadix;
#pragma unroll
      for (int j = 0; j < ITEMS; j++) {
        const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
        const bool ranked = pos < n;
        const uint32_t d = ranked ? (key[j] >> shift) & 0xffu : kNotRanked;
        const uint32_t peers = nbits >= 8 ? peers_of(d, ranked) : peers_of_code(ranked ? s_code[(shift / 8) * kRadix + d] : 0u, ranked, nbits);
        const int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (lane == leader && d != kNotRanked) {
          old = h[d];
          h[d] = old + (uint32_t)__popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[j] = old + (uint32_t)__popc(peers & lt);
        __syncwarp();
      }
    }
    __syncthreads();
    // Each digit's counts made exclusive over the warps: thread (q, d) takes
    // warps [8q, 8q + 8), then adds the earlier groups' totals
    constexpr int kGroups = THREADS / kRadix;
    const int q = tid / kRadix, dg = tid % kRadix;
    uint32_t part = 0;
#pragma unroll
    for (int w = q * 8; w < q * 8 + 8; w++) {
      const uint32_t c = s_whist[w * kRadix + dg];
      s_whist[w * kRadix + dg] = part;
      part += c;
    }
    s_part[q * kRadix + dg] = part;
    __syncthreads();
    uint32_t total = 0, before = 0;
#pragma unroll
    for (int g = 0; g < kGroups; g++) {
      const uint32_t v = s_part[g * kRadix + dg];
      before += g < q ? v : 0u;
      total += v;
    }
    if (q > 0) {
#pragma unroll
      for (int w = q * 8; w < q * 8 + 8; w++) s_whist[w * kRadix + dg] += before;
    }
    if (tid < kRadix) s_cnt[tid] = total;
    const uint32_t st = digit_exclusive_scan<THREADS>(tid < kRadix ? total : 0u, s_wsum);
    if (tid < kRadix) s_start[tid] = st;
    __syncthreads();
    return n;
  };

  // Every place ranks with 8 ballots but the top one, whose histogram the
  // counting kernel built: a place of k distinct digits (the top byte of depth
  // keys: a few exponents) ranks on a compact code with ceil(log2 k) ballots
  if (tid < kMaxPasses) s_wsum[9 + tid] = 8u;
  int passes = a.passes;
  {
    const int top = a.passes - 1;
    const bool present = tid < kRadix && a.hist[top * kRadix + tid] != 0u;
    const uint32_t code = digit_exclusive_scan<THREADS>(present ? 1u : 0u, s_wsum);
    if (tid < kRadix) s_code[top * kRadix + tid] = code;
    const int distinct = __syncthreads_count(present);
    if (tid == 0) s_wsum[9 + top] = distinct <= 1 ? 0u : (uint32_t)(32 - __clz(distinct - 1));
    // Every valid key has the same top digit (depths within one top-byte range): the top pass
    // would keep the order, so the pass before it writes the outputs
    if (distinct == 1 && passes > 1) passes--;
  }

  for (int place = 0; place < passes; place++) {
    const int shift = 8 * place;
    const bool last = place == passes - 1;
    const bool to_a = a.drop ? (place & 1) != 0 : (place & 1) == 0;
    uint32_t* kout = last ? a.keys_out : (to_a ? a.keys_a : a.keys_b);
    uint32_t* vout = last ? a.vals_out : (to_a ? a.vals_a : a.vals_b);

    // The block's digit counts of this pass
    if (tid < kRadix) s_blk[tid] = 0;
    for (uint32_t sub = 0; sub < nsub; sub++) {
      load_rank(sub, shift, nsub == 1);
      if (tid < kRadix) s_blk[tid] += s_cnt[tid];
    }
    __syncthreads();
    if (tid < kRadix) __stcg(&a.block_counts[(size_t)b * kRadix + tid], s_blk[tid]);
    barriers++;
    grid_barrier(a, barriers * G, !(place == a.silent_pass && b == 0));

    // Offsets: the digit's start in the segment plus the earlier blocks' counts of it
    {
      constexpr int kQuarters = THREADS >= 4 * kRadix ? 4 : THREADS / kRadix;
      const int q = tid / kRadix, d = tid % kRadix;
      // every block's count of the digit (its total) and the earlier blocks'; the
      // exchange buffer is free until the scatter and holds the totals' partial sums
      if (q < kQuarters) {
        uint32_t sum = 0, all = 0;
        const uint32_t per = (G + kQuarters - 1) / kQuarters;
        const uint32_t from = min((uint32_t)q * per, G), to = min(from + per, G);
#pragma unroll 8
        for (uint32_t e = from; e < to; e++) {
          const uint32_t c = __ldcg(&a.block_counts[(size_t)e * kRadix + d]);
          all += c;
          sum += e < b ? c : 0u;
        }
        s_part[q * kRadix + d] = sum;
        s_exchange[q * kRadix + d] = all;
      }
      __syncthreads();
      uint32_t total = 0;
      if (tid < kRadix) {
#pragma unroll
        for (int k = 0; k < kQuarters; k++) total += s_exchange[k * kRadix + tid];
      }
      const uint32_t digit_start = digit_exclusive_scan<THREADS>(total, s_wsum);
      if (tid < kRadix) {
        uint32_t before = 0;
#pragma unroll
        for (int k = 0; k < kQuarters; k++) before += s_part[k * kRadix + tid];
        s_base[tid] = (uint32_t)seg_begin + digit_start + before;
      }
      __syncthreads();
    }

    // Scatter, sub-tile by sub-tile in order
    const uint32_t seg_end = (uint32_t)seg_begin + V;
    for (uint32_t sub = 0; sub < nsub; sub++) {
      const uint32_t n = nsub == 1 ? min(kSub, len) : load_rank(sub, shift, true);
      const uint64_t start = seg_begin + lo + (uint64_t)sub * kSub;
      const bool busy = warp_base < n;  // the warp holds keys of this sub-tile
      if (busy) {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
          const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
          if (pos < n) {
            const uint32_t dj = (key[j] >> shift) & 0xffu;
            rank[j] += s_start[dj] + s_whist[warp * kRadix + dj];
            s_exchange[rank[j]] = key[j];
          } else {
            rank[j] = 0xffffffffu;
          }
        }
      }
      __syncthreads();
      uint32_t dest[ITEMS];
#pragma unroll
      for (int k = 0; k < ITEMS; k++) {
        const uint32_t i = (uint32_t)k * THREADS + tid;
        dest[k] = 0xffffffffu;
        if ((uint32_t)k * THREADS < n && i < n) {
          const uint32_t kk = s_exchange[i];
          const uint32_t dd = (kk >> shift) & 0xffu;
          const uint32_t dst = s_base[dd] + (i - s_start[dd]);
          if (dst >= (uint32_t)seg_begin && dst < seg_end) {  // in bounds even if a wait gave up
            dest[k] = dst;
            if (kout) kout[dst] = kk;
          } else {
            check_failed(a.error_flag);
          }
        }
      }
      if (vin) asm volatile("cp.async.wait_all;" ::: "memory");
      __syncthreads();
      const bool vec = vin && (reinterpret_cast<uintptr_t>(vin + start) & 15u) == 0;
      const uint32_t staged = vec ? (n & ~3u) : 0u;
      if (busy) {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
          if (rank[j] != 0xffffffffu) {
            const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
            const uint32_t v = !vin ? (uint32_t)(start - seg_begin) + pos
                                    : (pos < staged ? s_vals[pos] : __ldcg(&vin[start + pos]));
            s_exchange[rank[j]] = v;
          }
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < ITEMS; k++) {
        if ((uint32_t)k * THREADS < n && dest[k] != 0xffffffffu) vout[dest[k]] = s_exchange[(uint32_t)k * THREADS + tid];
      }
      if (tid < kRadix) s_base[tid] += s_cnt[tid];
      __syncthreads();
    }
    if (!last) {
      barriers++;
      grid_barrier(a, barriers * G, true);
    }
    kin = kout;
    vin = vout;
  }
}

// The cooperative variants: threads per block and keys per thread of a sub-tile
using CoopKernel = void (*)(CoopArgs);
struct CoopVariant {
  CoopKernel fn;
  int threads;
  size_t smem;
};

CoopVariant coop_variant(int id) {
  switch (id) {
    case kCoop512x16: return {k_sort_coop<512, 16>, 512, CoopShape<512, 16>::kBytes};
    case kCoop1024x8: return {k_sort_coop<1024, 8>, 1024, CoopShape<1024, 8>::kBytes};
    default: return {k_sort_coop<1024, 16>, 1024, CoopShape<1024, 16>::kBytes};
  }
}

}  // namespace

// Blocks of a variant resident on the current device (0: it cannot launch
// cooperatively), found once per device and variant
int coop_blocks(int id) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({device, id});
    if (it != cache.end()) return it->second;
  }
  const CoopVariant v = coop_variant(id);
  int sms = 0, per_sm = 0, coop = 0;
  int blocks = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) == cudaSuccess && coop &&
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
      cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem) == cudaSuccess &&
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.fn, v.threads, v.smem) == cudaSuccess) {
    blocks = sms * std::min(per_sm, 1024 / v.threads);
  }
  cudaGetLastError();
  std::lock_guard<std::mutex> lock(mu);
  cache[{device, id}] = blocks;
  return blocks;
}

uint32_t sort_small_pass_tiles(uint32_t max_tiles) {
  return max_tiles <= kSmallSortTiles ? max_tiles * (uint32_t)(kSortItems / kSmallItems) : 0u;
}

size_t sort_small_state_words(int segments, int passes, uint32_t max_tiles) {
  // hist [S][passes][256], valid [S], ref_hidden [S], counters [passes + 1], tile_valid [max_tiles]
  return (size_t)segments * passes * kRadix + 2 * (size_t)segments + (size_t)passes + 1 + max_tiles;
}

cudaError_t sort_segments(const SortCall& c, cudaStream_t stream, int* launches) {
  const int passes = c.bits / 8;
  const uint32_t mask = c.bits == 32 ? 0xffffffffu : ((1u << c.bits) - 1u);
  // The reference's visible count: keys whose top digit of its own layout is all ones
  const int ref_shift = c.bits == 16 ? 0 : (c.bits == 24 ? 11 : 16);
  const uint32_t ref_top = c.bits == 24 ? 0x1fffu : 0xffffu;
  const SortScratch& sc = c.scratch;
  if (c.segs.max_tiles == 0) {
    return c.visible ? cudaMemsetAsync(c.visible, 0, (size_t)c.segs.count * 4, stream) : cudaSuccess;
  }
  // In place (a WgpuRadixSort): the partition may not write the tail while
  // other tiles still read there, so the largest key is ranked like any other
  const int drop = c.keys_out != c.keys_in && c.vals_out != c.vals_in && !c.no_drop ? 1 : 0;
  int n_launch = 0;
  cudaError_t err;
  if (!c.zeroed) {
    err = cudaMemsetAsync(sc.hist, 0, sort_small_state_words(c.segs.count, passes, c.segs.max_tiles) * 4, stream);
    if (err != cudaSuccess) return err;
  }
  // One segment may take the cooperative digit passes, which need only the top place's histogram
  const int n_coop = c.coop != kCoopNone && c.segs.count == 1 && sc.block_counts ? coop_blocks(c.coop) : 0;
  const bool coop = n_coop > 0 && (uint32_t)n_coop <= kMaxCoopBlocks;
  using CountKernel = void (*)(const uint32_t*, uint32_t, int, uint32_t, int, SortSegments, uint32_t*, uint32_t*,
                               uint32_t*, uint32_t*, uint32_t*);
  const CountKernel count = passes == 2 ? (coop ? k_sort_count<2, true> : k_sort_count<2, false>)
                            : passes == 3 ? (coop ? k_sort_count<3, true> : k_sort_count<3, false>)
                                          : (coop ? k_sort_count<4, true> : k_sort_count<4, false>);
  err = launch_after(count, c.segs.max_tiles, kSortThreads, 0, stream, c.keys_in, mask, ref_shift, ref_top, drop, c.segs,
                     sc.hist, sc.valid, sc.ref_hidden, sc.tile_valid, c.epoch);
  if (err != cudaSuccess) return err;
  n_launch++;
  // After a partition the digit passes may take shorter tiles (c.pass_items
  // keys a thread; 0: 1024-key tiles for small sorts, else 4096): a pass's
  // time is then one short tile's chain, when the lookback words hold the
  // extra tiles. Without the partition the passes keep the 4096-key tiles of
  // the segments as given.
  int items = kSortItems;
  if (drop) {
    const int want = c.pass_items ? c.pass_items : (sort_small_pass_tiles(c.segs.max_tiles) ? kSmallItems : kSortItems);
    const uint32_t tiles = c.segs.max_tiles * (uint32_t)(kSortItems / want);
    if ((want == 4 || want == 8 || want == 16) && (uint64_t)passes * tiles * kRadix <= c.lookback_words) items = want;
  }
  const uint32_t pass_tiles = c.segs.max_tiles * (uint32_t)(kSortItems / items);
  // Without the partition every key is valid: the digit passes use the segments as given
  SortSegments vsegs = drop ? SortSegments{sc.vbegin, sc.vend, sc.vtiles, c.segs.count, pass_tiles} : c.segs;

  PassArgs a{};
  a.key_mask = mask;
  a.hist = sc.hist;
  a.passes = passes;
  a.epoch = c.epoch;
  a.error_flag = c.error_flag;
  a.spin_limit = c.spin_limit ? c.spin_limit : kSpinLimit;
  const uint32_t* ki = c.keys_in;
  const uint32_t* vi = c.vals_in;
  if (drop) {
    // Valid keys packed into the A buffers, the largest keys to the outputs' tails
    PartArgs p{};
    p.keys_in = c.keys_in;
    p.vals_in = c.vals_in;
    p.keys_front = sc.keys_a;
    p.vals_front = sc.vals_a;
    p.tail_keys = c.keys_out;
    p.tail_vals = c.vals_out;
    p.key_mask = mask;
    p.segs = c.segs;
    p.valid_count = sc.valid;
    p.tile_valid = sc.tile_valid;
    p.counter = sc.counters + passes;
    p.vbegin = sc.vbegin;
    p.vend = sc.vend;
    p.vtiles = sc.vtiles;
    p.pass_tile = (uint32_t)(kSortThreads * items);
    p.error_flag = c.error_flag;
    p.visible = c.visible;
    p.ref_hidden = c.visible_ref ? sc.ref_hidden : nullptr;
    err = launch_after(k_partition, c.segs.max_tiles, kSortThreads, 0, stream, p);
    if (err != cudaSuccess) return err;
    n_launch++;
    ki = sc.keys_a;
    vi = sc.vals_a;
  }
  if (coop) {
    // A block a 4096-key tile of the sort's capacity, up to every SM slot: a
    // small sort's passes then wait on fewer blocks at their grid barriers and
    // sum fewer blocks' counts
    const int blocks = (int)std::min<uint32_t>((uint32_t)n_coop, std::max<uint32_t>(1u, c.segs.max_tiles));
    {
      const CoopVariant v = coop_variant(c.coop);
      CoopArgs ca{};
      ca.keys_in = ki;
      ca.vals_in = vi;
      ca.keys_a = sc.keys_a;
      ca.vals_a = sc.vals_a;
      ca.keys_b = sc.keys_b;
      ca.vals_b = sc.vals_b;
      ca.keys_out = c.keys_out;
      ca.vals_out = c.vals_out;
      ca.begin = vsegs.begin;
      ca.end = vsegs.end;
      ca.hist = sc.hist;
      ca.block_counts = sc.block_counts;
      ca.barrier = sc.counters;  // the first pass's tile counter, which the onesweep would use (zeroed per sort)
      ca.error_flag = c.error_flag;
      ca.key_mask = mask;
      ca.passes = passes;
      ca.drop = drop;
      ca.spin_limit = a.spin_limit;
      ca.silent_pass = c.silent_pass;
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3((unsigned)blocks);
      cfg.blockDim = dim3((unsigned)v.threads);
      cfg.dynamicSmemBytes = v.smem;
      cfg.stream = stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      err = cudaLaunchKernelEx(&cfg, v.fn, ca);
      if (err != cudaSuccess) return err;
      n_launch++;
      if (!drop && c.visible) {
        err = launch_visible(c.segs.begin, c.segs.end, c.visible_ref ? sc.ref_hidden : nullptr, sc.valid, c.segs.count,
                             c.visible, stream);
        if (err != cudaSuccess) return err;
        n_launch++;
      }
      if (launches) *launches += n_launch;
      return cudaGetLastError();
    }
  }
  for (int place = 0; place < passes; place++) {
    const bool last = place == passes - 1;
    // Ping-pong: after the partition the passes read A, B, A, ...; without it the first reads the input
    const bool to_a = drop ? place % 2 == 1 : place % 2 == 0;
    a.keys_in = ki;
    a.vals_in = vi;
    a.keys_out = last ? c.keys_out : (to_a ? sc.keys_a : sc.keys_b);
    a.vals_out = last ? c.vals_out : (to_a ? sc.vals_a : sc.vals_b);
    a.shift = 8 * place;
    a.segs = vsegs;
    a.place = place;
    a.lookback = c.lookback + (size_t)place * pass_tiles * kRadix;
    a.counter = sc.counters + place;
    a.silent_tile = place == c.silent_pass ? 0u : ~0u;
    const bool first = place == 0 && !drop;
    const bool keys = !(last && a.keys_out == nullptr);
    void (*kernel)(PassArgs) =
        first ? k_onesweep<true, true, kSortItems>
        : items == 4 ? (keys ? k_onesweep<false, true, 4> : k_onesweep<false, false, 4>)
        : items == 8 ? (keys ? k_onesweep<false, true, 8> : k_onesweep<false, false, 8>)
                     : (keys ? k_onesweep<false, true, kSortItems> : k_onesweep<false, false, kSortItems>);
    err = launch_after(kernel, pass_tiles, kSortThreads, 0, stream, a);
    if (err != cudaSuccess) return err;
    n_launch++;
    ki = a.keys_out;
    vi = a.vals_out;
  }
  if (!drop && c.visible) {
    err = launch_visible(c.segs.begin, c.segs.end, c.visible_ref ? sc.ref_hidden : nullptr, sc.valid, c.segs.count,
                         c.visible, stream);
    if (err != cudaSuccess) return err;
    n_launch++;
  }
  if (launches) *launches += n_launch;
  return cudaGetLastError();
}

}  // namespace rdx
