// Sort keys from distances, order-preserving compaction, and the small
// device-side helpers of indirect sorts and the splat sorter.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t key_f64(double v, int bits) {
  return key_of_bits(__float_as_uint(__double2float_rn(v)), bits);
}

__device__ __forceinline__ uint32_t key_f32(float v, int bits) {
  if (!(v > 0.0f) && !isnan(v)) v = 0.0f;  // max(distance, 0)
  return key_of_bits(__float_as_uint(v), bits);
}

// VEC: four distances a thread per step, read and written as 16-byte vectors
// (both buffers 16-byte aligned); the n % 4 tail by the first threads
template <bool VEC>
__global__ void k_keys_f64(const double* __restrict__ d, uint64_t n, int bits, uint32_t* __restrict__ keys) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nv = VEC ? n / 4 : 0;
  if constexpr (VEC) {
    for (uint64_t i = t; i < nv; i += stride) {
      const double2 a = __ldcs(reinterpret_cast<const double2*>(d) + 2 * i);
      const double2 b = __ldcs(reinterpret_cast<const double2*>(d) + 2 * i + 1);
      __stcs(reinterpret_cast<uint4*>(keys) + i,
             make_uint4(key_f64(a.x, bits), key_f64(a.y, bits), key_f64(b.x, bits), key_f64(b.y, bits)));
    }
  }
  for (uint64_t i = nv * 4 + t; i < n; i += stride) keys[i] = key_f64(d[i], bits);
}

template <bool VEC>
__global__ void k_keys_f32(const float* __restrict__ d, uint64_t n, int bits, uint32_t* __restrict__ keys) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nv = VEC ? n / 4 : 0;
  if constexpr (VEC) {
    for (uint64_t i = t; i < nv; i += stride) {
      const float4 v = __ldcs(reinterpret_cast<const float4*>(d) + i);
      __stcs(reinterpret_cast<uint4*>(keys) + i,
             make_uint4(key_f32(v.x, bits), key_f32(v.y, bits), key_f32(v.z, bits), key_f32(v.w, bits)));
    }
  }
  for (uint64_t i = nv * 4 + t; i < n; i += stride) keys[i] = key_f32(d[i], bits);
}

__global__ void k_visible(const uint64_t* begin, const uint64_t* end, const uint32_t* ref_hidden,
                          const uint32_t* valid, int segments, uint32_t* visible) {
  pdl_wait();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < segments) visible[s] = ref_hidden ? (uint32_t)(end[s] - begin[s]) - ref_hidden[s] : valid[s];
}

__global__ void k_indirect_segments(const uint32_t* count, uint64_t capacity, uint64_t* begin, uint64_t* end,
                                    uint32_t* tiles) {
  const uint64_t c = min((uint64_t)*count, capacity);
  begin[0] = 0;
  end[0] = c;
  tiles[0] = 0;
  tiles[1] = (uint32_t)((c + kSortTile - 1) / kSortTile);
}

__global__ void k_draw_args(const uint32_t* count, uint32_t* args) {
  // drawIndexedIndirect: 1024 quads of 6 indices per instance (WgpuSplatSorter.ts:46-57)
  args[0] = 1024u * 6u;
  args[1] = (*count + 1023u) / 1024u;
  args[2] = 0;
  args[3] = 0;
  args[4] = 0;
}

constexpr int kCompactItems = 16;
constexpr int kCompactTile = kThreads * kCompactItems;
constexpr int kScanThreads = 1024;

// Order-preserving compaction (WgpuCompact.ts:22-132) in three kernels: each
// tile's valid count, one block's exclusive scan of those counts, and the
// scatter, whose tiles take their offsets from the scan and wait on no other
// tile (a single pass chaining the tiles by decoupled lookback ran at half
// the speed: every tile then waits on its predecessors' counts).

// Valid keys of each 4096-key tile (one block a tile)
__global__ void __launch_bounds__(kThreads) k_compact_count(const uint32_t* __restrict__ keys, uint64_t n,
                                                            uint32_t invalid, uint32_t* __restrict__ tile_valid) {
  __shared__ uint32_t s_warp[kThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  pdl_wait();
  pdl_trigger();
  const uint64_t base = (uint64_t)blockIdx.x * kCompactTile + (uint64_t)warp * (kCompactItems * 32);
  uint32_t count = 0;
#pragma unroll
  for (int j = 0; j < kCompactItems; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    count += i < n && __ldg(&keys[i]) != invalid ? 1u : 0u;
  }
  count = __reduce_add_sync(0xffffffffu, count);
  if (lane == 0) s_warp[warp] = count;
  __syncthreads();
  if (tid == 0) {
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++) total += s_warp[w];
    tile_valid[blockIdx.x] = total;
  }
}

// Exclusive scan of the tiles' valid counts, in place (one block; a thread
// takes a run of consecutive tiles); the total is the valid count
__global__ void __launch_bounds__(kScanThreads) k_compact_scan(uint32_t* __restrict__ tile_valid, uint32_t tiles,
                                                               uint32_t* __restrict__ count_out) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  pdl_wait();
  pdl_trigger();
  const uint32_t per = (tiles + kScanThreads - 1) / kScanThreads;
  const uint32_t lo = min((uint32_t)tid * per, tiles), hi = min(lo + per, tiles);
  uint32_t sum = 0;
  for (uint32_t t = lo; t < hi; t++) sum += tile_valid[t];
  uint32_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;  // inclusive over the warps
  }
  __syncthreads();
  uint32_t run = (warp > 0 ? s_warp[warp - 1] : 0u) + x - sum;
  for (uint32_t t = lo; t < hi; t++) {
    const uint32_t c = tile_valid[t];
    tile_valid[t] = run;
    run += c;
  }
  if (tid == kScanThreads - 1) *count_out = run;  // the last run ends at the total
}

// The valid keys of a tile, in order, at the tile's offset; their indices beside them
__global__ void __launch_bounds__(kThreads) k_compact_scatter(const uint32_t* __restrict__ keys, uint64_t n,
                                                              uint32_t invalid, const uint32_t* __restrict__ tile_offset,
                                                              const uint32_t* __restrict__ count,
                                                              uint32_t* __restrict__ keys_out,
                                                              uint32_t* __restrict__ vals_out,
                                                              uint32_t* __restrict__ error_flag) {
  __shared__ uint32_t s_warp[kThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  pdl_wait();
  pdl_trigger();
  const uint64_t base = (uint64_t)blockIdx.x * kCompactTile + (uint64_t)warp * (kCompactItems * 32);
  uint32_t k[kCompactItems];
  uint32_t ballots[kCompactItems];
  uint32_t valid = 0;
#pragma unroll
  for (int j = 0; j < kCompactItems; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    k[j] = i < n ? __ldg(&keys[i]) : invalid;
    ballots[j] = __ballot_sync(0xffffffffu, i < n && k[j] != invalid);
    valid += (uint32_t)__popc(ballots[j]);
  }
  if (lane == 0) s_warp[warp] = valid;
  __syncthreads();
  uint32_t at = tile_offset[blockIdx.x];
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) at += w < warp ? s_warp[w] : 0u;
  const uint32_t total = min(*count, (uint32_t)min(n, (uint64_t)0xffffffffu));
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kCompactItems; j++) {
    if (ballots[j] & (1u << lane)) {
      const uint32_t p = at + (uint32_t)__popc(ballots[j] & lt);
      if (p >= total) {
        check_failed(error_flag);
        continue;
      }
      keys_out[p] = k[j];
      vals_out[p] = (uint32_t)(base + (uint64_t)j * 32 + lane);
    }
    at += (uint32_t)__popc(ballots[j]);
  }
}

// Blocks for n items a thread each, at most `cap` (a grid-stride loop takes the rest)
int grid_for(uint64_t n, uint64_t cap) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g > cap) g = cap;
  return (int)(g > 0 ? g : 1);
}

constexpr uint64_t kKeyBlocks = 148ull * 16;  // 16 blocks of 256 threads an SM

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

cudaError_t launch_keys_f64(const double* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (aligned16(d) && aligned16(keys)) {
    k_keys_f64<true><<<grid_for(n / 4 + 1, kKeyBlocks), kThreads, 0, s>>>(d, n, bits, keys);
  } else {
    k_keys_f64<false><<<grid_for(n, kKeyBlocks), kThreads, 0, s>>>(d, n, bits, keys);
  }
  return cudaGetLastError();
}

cudaError_t launch_keys_f32(const float* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  if (aligned16(d) && aligned16(keys)) {
    k_keys_f32<true><<<grid_for(n / 4 + 1, kKeyBlocks), kThreads, 0, s>>>(d, n, bits, keys);
  } else {
    k_keys_f32<false><<<grid_for(n, kKeyBlocks), kThreads, 0, s>>>(d, n, bits, keys);
  }
  return cudaGetLastError();
}

cudaError_t launch_visible(const uint64_t* begin, const uint64_t* end, const uint32_t* ref_hidden,
                           const uint32_t* valid, int segments, uint32_t* visible, cudaStream_t s) {
  return launch_after(k_visible, (segments + 127) / 128, 128, 0, s, begin, end, ref_hidden, valid, segments, visible);
}

cudaError_t launch_compact(const uint32_t* keys, uint64_t n, uint32_t invalid, uint32_t* keys_out, uint32_t* vals_out,
                           uint32_t* count_out, uint32_t* tile_valid, uint32_t* error_flag, cudaStream_t s) {
  if (n == 0) return cudaMemsetAsync(count_out, 0, 4, s);
  const uint32_t tiles = (uint32_t)((n + kCompactTile - 1) / kCompactTile);
  cudaError_t err = launch_after(k_compact_count, tiles, kThreads, 0, s, keys, n, invalid, tile_valid);
  if (err != cudaSuccess) return err;
  err = launch_after(k_compact_scan, 1, kScanThreads, 0, s, tile_valid, tiles, count_out);
  if (err != cudaSuccess) return err;
  return launch_after(k_compact_scatter, tiles, kThreads, 0, s, keys, n, invalid, (const uint32_t*)tile_valid,
                      (const uint32_t*)count_out, keys_out, vals_out, error_flag);
}

cudaError_t launch_indirect_segments(const uint32_t* count, uint64_t capacity, uint64_t* begin, uint64_t* end,
                                     uint32_t* tiles, cudaStream_t s) {
  k_indirect_segments<<<1, 1, 0, s>>>(count, capacity, begin, end, tiles);
  return cudaGetLastError();
}

cudaError_t launch_draw_args(const uint32_t* count, uint32_t* args, cudaStream_t s) {
  k_draw_args<<<1, 1, 0, s>>>(count, args);
  return cudaGetLastError();
}

}  // namespace rdx
