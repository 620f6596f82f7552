// Sort keys from distances, order-preserving compaction, and the small
// device-side helpers of indirect sorts and the splat sorter.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {

namespace {

constexpr int kThreads = 256;

__global__ void k_keys_f64(const double* __restrict__ d, uint64_t n, int bits, uint32_t* __restrict__ keys) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = key_of_bits(__float_as_uint(__double2float_rn(d[i])), bits);
  }
}

__global__ void k_keys_f32(const float* __restrict__ d, uint64_t n, int bits, uint32_t* __restrict__ keys) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float v = d[i];
    if (!(v > 0.0f) && !isnan(v)) v = 0.0f;  // max(distance, 0)
    keys[i] = key_of_bits(__float_as_uint(v), bits);
  }
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

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int kCompactItems = 16;
constexpr int kCompactTile = kThreads * kCompactItems;

// Order-preserving compaction (WgpuCompact.ts:22-132) in one pass: tiles in
// launch order (a tile counter), the valid count of each tile chained by
// decoupled lookback. lookback[0] is the tile counter, lookback[1 + t] tile t.
__global__ void __launch_bounds__(kThreads) k_compact(const uint32_t* __restrict__ keys, uint64_t n, uint32_t invalid,
                                                      uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
                                                      uint32_t* __restrict__ count_out, uint32_t* __restrict__ lookback,
                                                      uint32_t* __restrict__ error_flag) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kThreads / 32 + 1];
  __shared__ uint32_t s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(&lookback[0], 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kCompactTile + (uint64_t)warp * (kCompactItems * 32);
  uint32_t k[kCompactItems];
  uint32_t ballots[kCompactItems];
  uint32_t count = 0;
#pragma unroll
  for (int j = 0; j < kCompactItems; j++) {
    const uint64_t i = base + (uint64_t)j * 32 + lane;
    k[j] = i < n ? __ldg(&keys[i]) : invalid;
    ballots[j] = __ballot_sync(0xffffffffu, i < n && k[j] != invalid);
    count += (uint32_t)__popc(ballots[j]);
  }
  if (lane == 0) s_warp[warp] = count;
  __syncthreads();
  if (tid == 0) {
    uint32_t sum = 0;
    for (int w = 0; w < kThreads / 32; w++) {
      const uint32_t c = s_warp[w];
      s_warp[w] = sum;
      sum += c;
    }
    s_warp[kThreads / 32] = sum;
    const uint32_t flag_agg = 1u << 30, flag_inc = 2u << 30, flags = 3u << 30;
    uint32_t prefix = 0;
    if (tile == 0) {
      st_relaxed(&lookback[1], flag_inc | sum);
    } else {
      st_relaxed(&lookback[1 + tile], flag_agg | sum);
      uint32_t t = tile - 1, spins = 0;
      while (true) {
        const uint32_t v = ld_relaxed(&lookback[1 + t]);
        if ((v & flags) == 0) {
          if (++spins > kSpinLimit) {
            atomicOr(error_flag, kErrTimeout);
            break;
          }
          if (spins > 32) __nanosleep(32);
          continue;
        }
        prefix += v & ((1u << 30) - 1u);
        if ((v & flags) == flag_inc) break;
        t--;
      }
      st_relaxed(&lookback[1 + tile], flag_inc | (prefix + sum));
    }
    s_prefix = prefix;
    const uint64_t tiles = (n + kCompactTile - 1) / kCompactTile;
    if ((uint64_t)tile == tiles - 1) *count_out = prefix + sum;
  }
  __syncthreads();
  uint32_t at = s_prefix + s_warp[warp];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kCompactItems; j++) {
    if (ballots[j] & (1u << lane)) {
      const uint32_t p = at + (uint32_t)__popc(ballots[j] & lt);
      if ((uint64_t)p >= n) {  // only after a bounded wait gave up
        check_failed(error_flag);
        continue;
      }
      keys_out[p] = k[j];
      vals_out[p] = (uint32_t)(base + (uint64_t)j * 32 + lane);
    }
    at += (uint32_t)__popc(ballots[j]);
  }
}

int grid_for(uint64_t n) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g > 148ull * 32) g = 148ull * 32;
  return (int)(g > 0 ? g : 1);
}

}  // namespace

cudaError_t launch_keys_f64(const double* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_keys_f64<<<grid_for(n), kThreads, 0, s>>>(d, n, bits, keys);
  return cudaGetLastError();
}

cudaError_t launch_keys_f32(const float* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_keys_f32<<<grid_for(n), kThreads, 0, s>>>(d, n, bits, keys);
  return cudaGetLastError();
}

cudaError_t launch_visible(const uint64_t* begin, const uint64_t* end, const uint32_t* ref_hidden,
                           const uint32_t* valid, int segments, uint32_t* visible, cudaStream_t s) {
  return launch_after(k_visible, (segments + 127) / 128, 128, 0, s, begin, end, ref_hidden, valid, segments, visible);
}

cudaError_t launch_compact(const uint32_t* keys, uint64_t n, uint32_t invalid, uint32_t* keys_out, uint32_t* vals_out,
                           uint32_t* count_out, uint32_t* lookback, uint32_t* error_flag, cudaStream_t s) {
  const uint64_t tiles = (n + kCompactTile - 1) / kCompactTile;
  cudaError_t err = cudaMemsetAsync(lookback, 0, (tiles + 1) * 4, s);
  if (err != cudaSuccess) return err;
  if (n == 0) return cudaMemsetAsync(count_out, 0, 4, s);
  k_compact<<<(unsigned)tiles, kThreads, 0, s>>>(keys, n, invalid, keys_out, vals_out, count_out, lookback, error_flag);
  return cudaGetLastError();
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
