// Stable LSD radix sort of uint32 keys with uint32 values for sm_100a: an
// upfront histogram kernel (every digit place in one read of the keys), then
// one onesweep kernel per 8-bit digit place. Each onesweep tile ranks its
// keys with warp match-based multisplit in shared memory, publishes its digit
// counts and finds its global offsets by decoupled lookback (single pass, no
// separate scan kernel), then scatters keys and values through shared memory
// so that writes of one digit run are contiguous.
//
// Replaces WgpuRadixSort (src/wgpu/WgpuRadixSort.ts:43-361: 3 dispatches per
// pass, histogram / scanBlocks / scatter with 8 one-bit splits) and
// SortKeys.sort (src/core/sort.ts:64-163). Any stable ascending sort yields the
// order of those two; the digit width here is the reference GPU sort's 8 bits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagInclusive = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1u;

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Segment holding `tile` (seg_tiles is non-decreasing, seg_tiles[0] = 0)
__device__ __forceinline__ int segment_of(const uint32_t* seg_tiles, int count, uint32_t tile) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (seg_tiles[mid] <= tile) {
      lo = mid;
    } else {
      hi = mid - 1;
    }
  }
  return lo;
}

// Exclusive scan over the 256 threads of a block (64-bit lanes); `sums` is
// 8 words of shared memory. Returns the thread's exclusive prefix.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint64_t s = lane < kSortWarps ? sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < kSortWarps; o <<= 1) {
      uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kSortWarps) sums[lane] = s;  // inclusive warp totals
  }
  __syncthreads();
  uint64_t before = warp > 0 ? sums[warp - 1] : 0;
  return before + x - v;
}

// ---- upfront histogram: every digit place of every segment, one read ----

template <int PASSES>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(
    const uint32_t* __restrict__ keys, uint32_t key_mask, int ref_shift, uint32_t ref_top,
    SortSegments segs, int tiles_per_block, uint32_t* __restrict__ hist,
    uint32_t* __restrict__ ref_hidden, uint32_t* __restrict__ lookback) {
  __shared__ uint32_t sh[PASSES][kRadix];
  __shared__ uint32_t s_hidden;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const uint32_t total_tiles = segs.seg_tiles[segs.count];
  const uint32_t tile0 = blockIdx.x * (uint32_t)tiles_per_block;
  if (tile0 >= total_tiles) return;
  const uint32_t tile_end = min(tile0 + (uint32_t)tiles_per_block, total_tiles);

#pragma unroll
  for (int p = 0; p < PASSES; p++) sh[p][tid] = 0;
  if (tid == 0) s_hidden = 0;
  __syncthreads();

  int seg = segment_of(segs.seg_tiles, segs.count, tile0);
  uint32_t hidden = 0;
  auto flush = [&](int s) {
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PASSES; p++) {
      uint32_t c = sh[p][tid];
      if (c) atomicAdd(&hist[((size_t)s * PASSES + p) * kRadix + tid], c);
      sh[p][tid] = 0;
    }
    uint32_t h = __reduce_add_sync(0xffffffffu, hidden);
    if (lane == 0 && h) atomicAdd(&s_hidden, h);
    hidden = 0;
    __syncthreads();
    if (tid == 0) {
      if (s_hidden) atomicAdd(&ref_hidden[s], s_hidden);
      s_hidden = 0;
    }
    __syncthreads();
  };

  for (uint32_t tile = tile0; tile < tile_end; tile++) {
    while (tile >= segs.seg_tiles[seg + 1]) {
      flush(seg);
      seg++;
    }
    // Zero this tile's lookback words of every pass (read by the onesweep kernels)
#pragma unroll
    for (int p = 0; p < PASSES; p++) lookback[((size_t)p * segs.max_tiles + tile) * kRadix + tid] = 0u;
    const uint64_t seg_begin = segs.seg_off[seg];
    const uint64_t base = seg_begin + (uint64_t)(tile - segs.seg_tiles[seg]) * kSortTile;
    const uint32_t n = (uint32_t)min((uint64_t)kSortTile, segs.seg_off[seg + 1] - base);
#pragma unroll 4
    for (int j = 0; j < kSortItems; j++) {
      const uint32_t pos = (uint32_t)j * kSortThreads + tid;
      const bool valid = pos < n;
      const uint32_t active = __ballot_sync(0xffffffffu, valid);
      if (valid) {
        const uint32_t k = __ldg(&keys[base + pos]) & key_mask;
        hidden += (k >> ref_shift) == ref_top;
        const int leader = __ffs(active) - 1;
#pragma unroll
        for (int p = 0; p < PASSES; p++) {
          const uint32_t d = (k >> (8 * p)) & 0xffu;
          const uint32_t first = __shfl_sync(active, d, leader);
          if (__all_sync(active, d == first)) {
            if (lane == leader) atomicAdd(&sh[p][d], (uint32_t)__popc(active));
          } else {
            atomicAdd(&sh[p][d], 1u);
          }
        }
      }
    }
  }
  flush(seg);
}

// ---- onesweep: one digit place ----

template <bool FIRST, bool WRITE_KEYS>
__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, uint32_t key_mask, int shift,
    SortSegments segs, const uint32_t* __restrict__ hist, int passes, int place,
    uint32_t* __restrict__ lookback, uint32_t* __restrict__ counter, uint32_t* __restrict__ error_flag) {
  __shared__ uint32_t s_whist[kSortWarps][kRadix];
  __shared__ uint32_t s_exchange[kSortTile];
  __shared__ uint32_t s_tile_start[kRadix];
  __shared__ uint32_t s_dest[kRadix];
  __shared__ uint64_t s_sums[kSortWarps];
  __shared__ uint32_t s_tile;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;

  if (tid == 0) s_tile = atomicAdd(counter, 1u);
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) s_whist[w][tid] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t total_tiles = segs.seg_tiles[segs.count];
  if (tile >= total_tiles) return;  // an indirect sort sized for its capacity

  const int seg = segment_of(segs.seg_tiles, segs.count, tile);
  const uint32_t local_tile = tile - segs.seg_tiles[seg];
  const uint64_t seg_begin = segs.seg_off[seg];
  const uint64_t base = seg_begin + (uint64_t)local_tile * kSortTile;
  const uint32_t n = (uint32_t)min((uint64_t)kSortTile, segs.seg_off[seg + 1] - base);

  // Load: warp w holds tile positions [w * 512, (w + 1) * 512), item j at j * 32 + lane
  uint32_t key[kSortItems], val[kSortItems];
  const uint32_t warp_base = (uint32_t)warp * (kSortItems * 32);
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t pos = warp_base + (uint32_t)j * 32 + lane;
    if (pos < n) {
      key[j] = __ldg(&keys_in[base + pos]) & key_mask;
      val[j] = FIRST && vals_in == nullptr ? (uint32_t)(base - seg_begin) + pos : __ldg(&vals_in[base + pos]);
    } else {
      key[j] = 0xffffffffu;  // padding: digit 255, after every real key of the tile
      val[j] = 0;
    }
  }

  // Rank: items in position order, equal digits counted by their lowest lane
  uint32_t rank[kSortItems];  // rank within the warp's digit, then the local position
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t d = (key[j] >> shift) & 0xffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (lane == leader) {
      old = s_whist[warp][d];
      s_whist[warp][d] = old + (uint32_t)__popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[j] = old + (uint32_t)__popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();

  // Thread d owns digit d: warp counts -> exclusive over warps, tile total
  const uint32_t d = (uint32_t)tid;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = s_whist[w][d];
    s_whist[w][d] = total;
    total += c;
  }
  const uint32_t real = total - (d == 0xffu ? (uint32_t)kSortTile - n : 0u);
  uint32_t* my_word = &lookback[(size_t)tile * kRadix + d];
  st_relaxed(my_word, (local_tile == 0 ? kFlagInclusive : kFlagAggregate) | real);

  // Tile-local digit starts (low word) and the segment's digit offsets (high word) in one scan
  const uint32_t seg_count = hist[((size_t)seg * passes + place) * kRadix + d];
  const uint64_t both = block_exclusive_scan(((uint64_t)seg_count << 32) | total, s_sums);
  const uint32_t tile_start = (uint32_t)both;
  const uint32_t seg_digit = (uint32_t)(both >> 32);
  s_tile_start[d] = tile_start;

  // Decoupled lookback over this segment's earlier tiles, bounded
  uint32_t prefix = 0;
  if (local_tile > 0) {
    uint32_t t = tile - 1;
    uint32_t spins = 0;
    while (true) {
      const uint32_t v = ld_relaxed(&lookback[(size_t)t * kRadix + d]);
      const uint32_t flag = v & kFlagMask;
      if (flag == 0) {
        if (++spins > kSpinLimit) {
          atomicExch(error_flag, 1u);
          break;
        }
        if (spins > 32) __nanosleep(32);
        continue;
      }
      prefix += v & kCountMask;
      if (flag == kFlagInclusive) break;
      t--;
    }
    st_relaxed(my_word, kFlagInclusive | (prefix + real));
  }
  s_dest[d] = (uint32_t)seg_begin + seg_digit + prefix - tile_start;
  __syncthreads();

  // Local sort of the keys in shared memory
#pragma unroll
  for (int j = 0; j < kSortItems; j++) {
    const uint32_t dj = (key[j] >> shift) & 0xffu;
    rank[j] += s_tile_start[dj] + s_whist[warp][dj];
    s_exchange[rank[j]] = key[j];
  }
  __syncthreads();
  // Destinations stay inside the segment even if a bounded wait gave up
  const uint32_t seg_end = (uint32_t)segs.seg_off[seg + 1];
  uint32_t dest[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const uint32_t i = (uint32_t)k * kSortThreads + tid;
    const uint32_t kk = s_exchange[i];
    dest[k] = s_dest[(kk >> shift) & 0xffu] + i;
    if (i >= n || dest[k] >= seg_end || dest[k] < (uint32_t)seg_begin) dest[k] = 0xffffffffu;
    if (WRITE_KEYS && dest[k] != 0xffffffffu) keys_out[dest[k]] = kk;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; j++) s_exchange[rank[j]] = val[j];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItems; k++) {
    const uint32_t i = (uint32_t)k * kSortThreads + tid;
    if (dest[k] != 0xffffffffu) vals_out[dest[k]] = s_exchange[i];
  }
}

template <bool FIRST, bool WRITE_KEYS>
void launch_onesweep(const uint32_t* ki, const uint32_t* vi, uint32_t* ko, uint32_t* vo, uint32_t mask,
                     int place, const SortSegments& segs, const SortScratch& sc, int passes,
                     uint32_t* error_flag, cudaStream_t stream) {
  k_onesweep<FIRST, WRITE_KEYS><<<segs.max_tiles, kSortThreads, 0, stream>>>(
      ki, vi, ko, vo, mask, 8 * place, segs, sc.hist, passes, place,
      sc.lookback + (size_t)place * segs.max_tiles * kRadix, sc.counters + place, error_flag);
}

}  // namespace

size_t sort_small_state_words(int segments, int passes) {
  return (size_t)segments * passes * kRadix + (size_t)segments + (size_t)passes;
}

cudaError_t sort_segments(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                          uint32_t* vals_out, const SortSegments& segs, int bits,
                          const SortScratch& sc, uint32_t* error_flag, cudaStream_t stream) {
  const int passes = bits / 8;
  const uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
  // The reference's visible count: keys whose top digit of its own layout is all ones
  const int ref_shift = bits == 16 ? 0 : (bits == 24 ? 11 : 16);
  const uint32_t ref_top = bits == 24 ? 0x1fffu : 0xffffu;
  if (segs.max_tiles == 0) return cudaSuccess;

  // hist, ref_hidden and counters are contiguous
  cudaError_t err = cudaMemsetAsync(sc.hist, 0, sort_small_state_words(segs.count, passes) * 4, stream);
  if (err != cudaSuccess) return err;
  const int target_blocks = 148 * 4;
  int tpb = (int)((segs.max_tiles + target_blocks - 1) / target_blocks);
  if (tpb < 1) tpb = 1;
  const int hist_blocks = (int)((segs.max_tiles + tpb - 1) / tpb);
  switch (passes) {
    case 2:
      k_sort_hist<2><<<hist_blocks, kSortThreads, 0, stream>>>(keys_in, mask, ref_shift, ref_top, segs, tpb,
                                                              sc.hist, sc.ref_hidden, sc.lookback);
      break;
    case 3:
      k_sort_hist<3><<<hist_blocks, kSortThreads, 0, stream>>>(keys_in, mask, ref_shift, ref_top, segs, tpb,
                                                              sc.hist, sc.ref_hidden, sc.lookback);
      break;
    default:
      k_sort_hist<4><<<hist_blocks, kSortThreads, 0, stream>>>(keys_in, mask, ref_shift, ref_top, segs, tpb,
                                                              sc.hist, sc.ref_hidden, sc.lookback);
      break;
  }
  // Ping-pong: pass 0 from the input, the last pass into the output
  const uint32_t* ki = keys_in;
  const uint32_t* vi = vals_in;
  for (int place = 0; place < passes; place++) {
    const bool last = place == passes - 1;
    uint32_t* ko = last ? keys_out : (place % 2 == 0 ? sc.keys_a : sc.keys_b);
    uint32_t* vo = last ? vals_out : (place % 2 == 0 ? sc.vals_a : sc.vals_b);
    if (place == 0) {
      launch_onesweep<true, true>(ki, vi, ko, vo, mask, place, segs, sc, passes, error_flag, stream);
    } else if (last && ko == nullptr) {
      launch_onesweep<false, false>(ki, vi, ko, vo, mask, place, segs, sc, passes, error_flag, stream);
    } else {
      launch_onesweep<false, true>(ki, vi, ko, vo, mask, place, segs, sc, passes, error_flag, stream);
    }
    ki = ko;
    vi = vo;
  }
  return cudaGetLastError();
}

}  // namespace rdx
