// Fused per-splat projection for sm_100a: table decode, SH colour from the
// head (object space), object -> head transform, ewa projection per eye, the
// reference's words, float outputs, the back-to-front sort key and (for a
// frame) the histogram of the keys' digits for the sort that follows.
//
// Restates, fused: SplatProjector.build (src/render/SplatProjector.ts:153-194),
// SplatGenerator.fromSplats.withSh (src/gpu/splatGenerator.ts:152-158),
// GpuShReader.color/apply (src/gpu/sh.tsl.ts:255-266), transformCov
// (src/render/splatTransform.tsl.ts:120-140), prepareSplat / splatInView /
// culls (src/render/projection.tsl.ts:42-140), ewa.project
// (src/render/projections.tsl.ts:95-148) and SplatProjection.write
// (src/render/SplatProjection.ts:141-153).
//
// Structure: a persistent grid; each block walks its 128-splat tiles. A tile's
// columns are staged into shared memory by TMA bulk copies
// (cp.async.bulk + mbarrier), two stages deep, so HBM streams while the
// previous tile computes. Phase 1 (every splat): the centre in float64, the
// key distance and the centre culls; splats culled in every eye are finished
// there. Phase 2 (a compacted list of the rest): SH, covariance and ewa.
//
// Precision: the head-space centre, the key distance and the centre culls are
// float64 with explicitly rounded operations, so keys and cull decisions equal
// the float64 oracle's. SH, the 2D mean and the covariance chain are float64
// too: the conic's off-diagonal and rgb near its clamp cancel. The 2D
// covariance is factored as T T^T with T = J^T W R S (2 x 3):
// a = sum u0k^2 s_k^2, b = sum u0k u1k s_k^2, and det(T T^T) by Cauchy-Binet,
// the sum over column pairs (j, k) of (s_j s_k (u0 x u1)_l)^2 - non-negative
// terms, no a d - b^2 cancellation. Bounds, angles and words are float32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr int kTile = kProjTile;  // splats per tile = threads per block
constexpr int kStages = 2;
constexpr uint32_t kWaitLimit = 1u << 24;  // polls of a stage's mbarrier before giving up

template <int DEG>
struct ShCount {
  static constexpr int value = DEG == 0 ? 0 : (DEG == 1 ? 3 : (DEG == 2 ? 8 : (DEG == 3 ? 15 : 24)));
};

// Byte offsets of the columns of one tile in a shared-memory stage (all 16-aligned)
template <int LAYOUT, int DEG, int CDT>
struct Stage {
  static constexpr int K = ShCount<DEG>::value;
  static constexpr int kColorRow = (1 + K) * 3 * (CDT == RDX_DTYPE_F16 ? 2 : 4);
  static constexpr int kCenters = 0;
  static constexpr int kLogScales = kCenters + kTile * 12;
  static constexpr int kQuats = kLogScales + kTile * 12;
  static constexpr int kOpacities = kQuats + kTile * 16;
  static constexpr int kColors = kOpacities + kTile * 4;
  static constexpr int kRawBytes = kColors + (kTile * kColorRow + 15) / 16 * 16;
  static constexpr int kTexels = (K + 3) / 4;
  static constexpr int kExtA = 0;
  static constexpr int kExtB = kTile * 16;
  static constexpr int kExtSh = 2 * kTile * 16;
  static constexpr int kExtBytes = (2 + kTexels) * kTile * 16;
  static constexpr int kBytes = ((LAYOUT == RDX_LAYOUT_RAW ? kRawBytes : kExtBytes) + 127) / 128 * 128;
};

// The column copies of one tile: shared-memory offset, source, bytes
struct TileCopies {
  int n;
  int dst[8];
  const unsigned char* src[8];
  uint32_t bytes[8];
};

template <int LAYOUT, int DEG, int CDT>
__device__ __forceinline__ void tile_copies(const DevTable& t, uint64_t i0, uint32_t cnt, TileCopies& c) {
  using S = Stage<LAYOUT, DEG, CDT>;
  c.n = 0;
  auto add = [&](int dst, const void* base, uint32_t row) {
    c.dst[c.n] = dst;
    c.src[c.n] = reinterpret_cast<const unsigned char*>(base) + i0 * row;
    c.bytes[c.n] = cnt * row;
    c.n++;
  };
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    add(S::kCenters, t.centers, 12);
    add(S::kLogScales, t.log_scales, 12);
    add(S::kQuats, t.quats, 16);
    add(S::kOpacities, t.opacities, 4);
    add(S::kColors, t.colors, S::kColorRow);
  } else {
    add(S::kExtA, t.ext_a, 16);
    add(S::kExtB, t.ext_b, 16);
#pragma unroll
    for (int k = 0; k < S::kTexels; k++) add(S::kExtSh + k * kTile * 16, t.ext_sh[k], 16);
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Issue the bulk copies of a full, 16-byte aligned tile (one thread)
__device__ __forceinline__ void issue_tma(uint64_t* bar, unsigned char* stage, const TileCopies& c) {
  uint32_t total = 0;
  for (int k = 0; k < c.n; k++) total += c.bytes[k];
  const uint32_t b = smem_addr(bar);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(total) : "memory");
  for (int k = 0; k < c.n; k++) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(stage + c.dst[k])),
        "l"(c.src[k]), "r"(c.bytes[k]), "r"(b)
        : "memory");
  }
}

// Bounded wait for a stage's phase; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t b = smem_addr(bar);
  for (uint32_t i = 0; i < kWaitLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The tile copied by the block's threads: partial tiles, unaligned tables
__device__ __forceinline__ void manual_copy(unsigned char* stage, const TileCopies& c) {
  for (int k = 0; k < c.n; k++) {
    const uint32_t bytes = c.bytes[k];
    const unsigned char* src = c.src[k];
    unsigned char* dst = stage + c.dst[k];
    if ((bytes & 3u) == 0 && ((uintptr_t)src & 3u) == 0) {
      for (uint32_t w = threadIdx.x; w < bytes / 4; w += kTile)
        reinterpret_cast<uint32_t*>(dst)[w] = __ldg(reinterpret_cast<const unsigned int*>(src) + w);
    } else {
      for (uint32_t w = threadIdx.x; w < bytes / 2; w += kTile)
        reinterpret_cast<unsigned short*>(dst)[w] = __ldg(reinterpret_cast<const unsigned short*>(src) + w);
    }
  }
}

// The 3DGS basis of band `band` along unit (x, y, z) in float64
// (src/gpu/sh.tsl.ts:60-102, src/core/sh.ts:376-407), n values into `basis`
__device__ __forceinline__ int sh_basis_band(int band, double x, double y, double z, double* basis) {
  const double xx = x * x, yy = y * y, zz = z * z;
  if (band == 1) {
    basis[0] = -0.4886025 * y;
    basis[1] = 0.4886025 * z;
    basis[2] = -0.4886025 * x;
    return 3;
  }
  if (band == 2) {
    basis[0] = 1.0925484 * x * y;
    basis[1] = -1.0925484 * y * z;
    basis[2] = 0.3153916 * (2.0 * zz - xx - yy);
    basis[3] = -1.0925484 * x * z;
    basis[4] = 0.5462742 * (xx - yy);
    return 5;
  }
  if (band == 3) {
    basis[0] = -0.5900436 * y * (3.0 * xx - yy);
    basis[1] = 2.8906114 * x * y * z;
    basis[2] = -0.4570458 * y * (4.0 * zz - xx - yy);
    basis[3] = 0.3731763 * z * (2.0 * zz - 3.0 * xx - 3.0 * yy);
    basis[4] = -0.4570458 * x * (4.0 * zz - xx - yy);
    basis[5] = 1.4453057 * z * (xx - yy);
    basis[6] = -0.5900436 * x * (xx - 3.0 * yy);
    return 7;
  }
  const double zz7m1 = 7.0 * zz - 1.0, zz7m3 = 7.0 * zz - 3.0;
  basis[0] = 2.5033429 * x * y * (xx - yy);
  basis[1] = -1.7701308 * y * z * (3.0 * xx - yy);
  basis[2] = 0.9461747 * x * y * zz7m1;
  basis[3] = -0.6690465 * y * z * zz7m3;
  basis[4] = 0.1057855 * (zz * (35.0 * zz - 30.0) + 3.0);
  basis[5] = -0.6690465 * x * z * zz7m3;
  basis[6] = 0.4730873 * (xx - yy) * zz7m1;
  basis[7] = -1.7701308 * x * z * (xx - 3.0 * yy);
  basis[8] = 0.6258357 * (xx * (xx - 3.0 * yy) - yy * (3.0 * xx - yy));
  return 9;
}

template <int LAYOUT, int DEG, int CDT>
__device__ __forceinline__ void read_centre(const unsigned char* st, int j, float& x, float& y, float& z, float& opacity,
                                            float ls[3]) {
  using S = Stage<LAYOUT, DEG, CDT>;
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    const float* c = reinterpret_cast<const float*>(st + S::kCenters) + j * 3;
    const float* l = reinterpret_cast<const float*>(st + S::kLogScales) + j * 3;
    x = c[0];
    y = c[1];
    z = c[2];
    ls[0] = l[0];
    ls[1] = l[1];
    ls[2] = l[2];
    opacity = reinterpret_cast<const float*>(st + S::kOpacities)[j];
  } else {
    const uint4 A = reinterpret_cast<const uint4*>(st + S::kExtA)[j];
    const uint4 B = reinterpret_cast<const uint4*>(st + S::kExtB)[j];
    x = __uint_as_float(A.x);
    y = __uint_as_float(A.y);
    z = __uint_as_float(A.z);
    opacity = (float)(A.w >> 24) * (1.0f / 128.0f);
    ls[0] = half_bits_to_float(B.y);
    ls[1] = half_bits_to_float(B.y >> 16);
    ls[2] = half_bits_to_float(B.z);
  }
}

template <int LAYOUT, int DEG, int CDT>
__device__ __forceinline__ void read_quat(const unsigned char* st, int j, double q[4]) {
  using S = Stage<LAYOUT, DEG, CDT>;
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    const float4 v = reinterpret_cast<const float4*>(st + S::kQuats)[j];
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
    q[3] = v.w;
  } else {
    decode_quat_oct32_f64(reinterpret_cast<const uint4*>(st + S::kExtB)[j].w, q);
  }
}

// Base rgb + SH (float64) of splat j, clamped at 0 when the table has SH
template <int LAYOUT, int DEG, int CDT>
__device__ __forceinline__ void colour(const unsigned char* st, int j, double dx, double dy, double dz, int cap,
                                       double rgb[3]) {
  using S = Stage<LAYOUT, DEG, CDT>;
  constexpr int K = S::K;
  double acc[3] = {0.0, 0.0, 0.0};
  const double l2 = dx * dx + dy * dy + dz * dz;
  const double inv = l2 > 0.0 ? 1.0 / sqrt(l2) : 0.0;
  const double x = dx * inv, y = dy * inv, z = dz * inv;
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    const unsigned char* row = st + S::kColors + j * S::kColorRow;
    auto value = [&](int v) -> double {
      if constexpr (CDT == RDX_DTYPE_F16) {
        return (double)__half2float(reinterpret_cast<const __half*>(row)[v]);
      } else {
        return (double)reinterpret_cast<const float*>(row)[v];
      }
    };
    rgb[0] = value(0);
    rgb[1] = value(1);
    rgb[2] = value(2);
    if constexpr (K > 0) {
#pragma unroll
      for (int band = 1; band <= DEG; band++) {
        if (band <= cap) {
          double basis[9];
          const int nb = sh_basis_band(band, x, y, z, basis);
#pragma unroll
          for (int k = 0; k < 9; k++) {
            if (k < nb) {
              const int ci = band * band - 1 + k;
              acc[0] = fma(value(3 + ci * 3), basis[k], acc[0]);
              acc[1] = fma(value(4 + ci * 3), basis[k], acc[1]);
              acc[2] = fma(value(5 + ci * 3), basis[k], acc[2]);
            }
          }
        }
      }
    }
  } else {
    decode_ext_rgb_f64(reinterpret_cast<const uint4*>(st + S::kExtB)[j].x, rgb);
    if constexpr (K > 0) {
#pragma unroll
      for (int band = 1; band <= DEG; band++) {
        if (band <= cap) {
          double basis[9];
          const int nb = sh_basis_band(band, x, y, z, basis);
#pragma unroll
          for (int k = 0; k < 9; k++) {
            if (k < nb) {
              const int ci = band * band - 1 + k;
              const uint32_t* words = reinterpret_cast<const uint32_t*>(st + S::kExtSh + (ci >> 2) * kTile * 16) + j * 4;
              double c[3];
              decode_ext_rgb_f64(words[ci & 3], c);
              acc[0] = fma(c[0], basis[k], acc[0]);
              acc[1] = fma(c[1], basis[k], acc[1]);
              acc[2] = fma(c[2], basis[k], acc[2]);
            }
          }
        }
      }
    }
  }
  if constexpr (K > 0) {
    rgb[0] = fmax(rgb[0] + acc[0], 0.0);
    rgb[1] = fmax(rgb[1] + acc[1], 0.0);
    rgb[2] = fmax(rgb[2] + acc[2], 0.0);
  }
}

// Warp-aggregated shared-memory histogram increment: lanes sharing a digit add once
__device__ __forceinline__ void hist_add(uint32_t* h, uint32_t d, bool valid) {
  uint32_t active = __ballot_sync(0xffffffffu, valid);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int round = 0; round < 2; round++) {
    if (!active) break;
    const int leader = __ffs(active) - 1;
    const uint32_t dl = __shfl_sync(0xffffffffu, d, leader);
    const uint32_t m = __ballot_sync(0xffffffffu, valid && d == dl) & active;
    if (lane == leader) atomicAdd(&h[dl], (uint32_t)__popc(m));
    active &= ~m;
  }
  if (active & (1u << lane)) atomicAdd(&h[d], 1u);
}

struct PerEye {  // float64 centre culls of one splat in one eye (phase 1 -> 2)
  double ex, ey, ez, clx, cly, clw;
};

template <int LAYOUT, int DEG, int CDT, int EYES, bool HIST>
__global__ void __launch_bounds__(kTile) k_project(const ProjDesc* __restrict__ descs, int n_desc, uint32_t total_tiles,
                                                   ProjOutputs out, ProjHist hist, uint32_t* __restrict__ error_flag) {
  using S = Stage<LAYOUT, DEG, CDT>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t s_bar[kStages];
  __shared__ int s_manual[kStages];
  __shared__ ProjDesc sd;
  __shared__ int s_desc;
  __shared__ int s_abort;
  __shared__ uint16_t s_list[kTile];
  __shared__ int s_warp_count[kTile / 32];
  __shared__ uint32_t s_key[kTile];
  __shared__ uint32_t s_keyval[kTile];   // the valid key of a candidate
  __shared__ double s_centre[3][kTile];  // object-space centre of a candidate
  __shared__ PerEye s_eye[EYES][kTile];
  __shared__ uint8_t s_eye_ok[kTile];
  __shared__ uint32_t s_hist[HIST ? kMaxPasses : 1][kRadix];
  __shared__ uint32_t s_valid;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  unsigned char* stage[kStages] = {smem, smem + S::kBytes};

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s_bar[s])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_valid = 0;
  }
  if constexpr (HIST) {
    for (int w = tid; w < kMaxPasses * kRadix; w += kTile) (&s_hist[0][0])[w] = 0;
  }

  // tile t -> descriptor (objects are contiguous runs of tiles)
  auto desc_of = [&](uint32_t t) {
    int lo = 0, hi = n_desc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].first_tile <= t) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    return lo;
  };
  // fill stage s with tile t (thread 0)
  auto issue = [&](int s, uint32_t t) {
    const ProjDesc& D = descs[desc_of(t)];
    const uint64_t i0 = (uint64_t)(t - D.first_tile) * kTile;
    const uint32_t cnt = (uint32_t)min((uint64_t)kTile, D.count - i0);
    TileCopies c;
    tile_copies<LAYOUT, DEG, CDT>(D.table, i0, cnt, c);
    const bool tma = cnt == (uint32_t)kTile && D.tma_ok;
    s_manual[s] = tma ? 0 : 1;
    if (tma) issue_tma(&s_bar[s], stage[s], c);
  };

  __syncthreads();
  const uint32_t stride = gridDim.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      const uint32_t t = blockIdx.x + s * stride;
      if (t < total_tiles) issue(s, t);
    }
  }
  uint32_t parity[kStages] = {0u, 0u};
  int cur_desc = -1;
  int hist_seg = -1;

  for (uint32_t k = 0;; k++) {
    const uint32_t t = blockIdx.x + k * stride;
    if (t >= total_tiles) break;
    const int s = (int)(k % kStages);
    if (tid == 0) s_desc = desc_of(t);
    __syncthreads();
    if (s_desc != cur_desc) {
      if constexpr (HIST) {
        // a new sort segment: flush the block's histogram of the previous one
        if (hist_seg >= 0 && descs[s_desc].segment != hist_seg) {
          for (int w = tid; w < hist.passes * kRadix; w += kTile) {
            const uint32_t c = (&s_hist[0][0])[w];
            if (c) atomicAdd(&hist.hist[(size_t)hist_seg * hist.passes * kRadix + w], c);
            (&s_hist[0][0])[w] = 0;
          }
          if (tid == 0 && s_valid) {
            atomicAdd(&hist.valid[hist_seg], s_valid);
            s_valid = 0;
          }
        }
      }
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&descs[s_desc]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
      for (int w = tid; w < (int)(sizeof(ProjDesc) / 4); w += kTile) dst[w] = src[w];
      cur_desc = s_desc;
      __syncthreads();
      hist_seg = sd.segment;
    }
    const uint64_t i0 = (uint64_t)(t - sd.first_tile) * kTile;
    const int cnt = (int)min((uint64_t)kTile, sd.count - i0);
    unsigned char* st = stage[s];
    if (s_manual[s]) {
      TileCopies c;
      tile_copies<LAYOUT, DEG, CDT>(sd.table, i0, (uint32_t)cnt, c);
      manual_copy(st, c);
      __syncthreads();
    } else {
      const bool ok = mbar_wait(&s_bar[s], parity[s]);
      parity[s] ^= 1u;
      if (!ok) {
        atomicExch(error_flag, 2u);
        s_abort = 1;
      }
      __syncthreads();
      if (s_abort) return;  // every thread: the wait gave up (a TMA never completed)
    }
    const DevParams& p = sd.params;
    const int j = tid;
    const bool live = j < cnt;
    const uint64_t gi = sd.out_offset + i0 + (uint64_t)j;

    // ---- phase 1: every splat: centre, distance, centre culls ----
    bool candidate = false;
    uint32_t key = invalid_key(sd.sort_bits);
    if (live) {
      float cxf, cyf, czf, opac, ls[3];
      read_centre<LAYOUT, DEG, CDT>(st, j, cxf, cyf, czf, opac, ls);
      const double cx = cxf, cy = cyf, cz = czf;
      const double hx = affine_row(sd.a + 0, cx, cy, cz);
      const double hy = affine_row(sd.a + 4, cx, cy, cz);
      const double hz = affine_row(sd.a + 8, cx, cy, cz);
      const double distance = __dsqrt_rn(dadd(dadd(dmul(hx, hx), dmul(hy, hy)), dmul(hz, hz)));
      // prepareSplat's opacity (projection.tsl.ts:42-64) and cullInvisible (66-69)
      double op = opac;
      if (op > 1.0) {
        op = fmin(op * 4.0 - 3.0, 5.0);
        if (p.lod_inflate) op = 1.0;
      }
      // exp(2 ln s) underflows to 0 below ln s = -372.6: a degenerate (zero) covariance
      const bool degenerate = sd.degenerate || (ls[0] < -372.6f && ls[1] < -372.6f && ls[2] < -372.6f);
      const bool invisible = op <= 0.0 || op < (double)p.min_alpha || degenerate;
      bool guarded = true;
      if (p.sort_guard > 0.0f && !invisible) {
        // inSortGuard (projection.tsl.ts:145-155), cov form, float32
        double q[4];
        read_quat<LAYOUT, DEG, CDT>(st, j, q);
        float qx = (float)q[0], qy = (float)q[1], qz = (float)q[2], qw = (float)q[3];
        const float ql2 = qx * qx + qy * qy + qz * qz + qw * qw;
        const float qi = ql2 > 0.0f ? rsqrtf(ql2) : 0.0f;
        qx *= qi;
        qy *= qi;
        qz *= qi;
        qw = ql2 > 0.0f ? qw * qi : 1.0f;
        const float R[9] = {1.f - 2.f * (qy * qy + qz * qz), 2.f * (qx * qy - qw * qz), 2.f * (qx * qz + qw * qy),
                            2.f * (qx * qy + qw * qz), 1.f - 2.f * (qx * qx + qz * qz), 2.f * (qy * qz - qw * qx),
                            2.f * (qx * qz - qw * qy), 2.f * (qy * qz + qw * qx), 1.f - 2.f * (qx * qx + qy * qy)};
        float inflate = 1.0f;
        if (opac > 1.0f && p.lod_inflate) {
          const float o = fminf(opac * 4.0f - 3.0f, 5.0f);
          inflate = expf((o * o - 1.0f) * (1.0f / (3.0f * 2.718281828459045f)));
        }
        const float sx = expf(ls[0]) * inflate, sy = expf(ls[1]) * inflate, sz = expf(ls[2]) * inflate;
        float ext2 = 0.0f;
#pragma unroll
        for (int r = 0; r < 3; r++) {
          const float a0 = (float)sd.a[r * 4 + 0], a1 = (float)sd.a[r * 4 + 1], a2 = (float)sd.a[r * 4 + 2];
          const float g0 = (a0 * R[0] + a1 * R[3] + a2 * R[6]) * sx;
          const float g1 = (a0 * R[1] + a1 * R[4] + a2 * R[7]) * sy;
          const float g2 = (a0 * R[2] + a1 * R[5] + a2 * R[8]) * sz;
          ext2 = fmaxf(ext2, g0 * g0 + g1 * g1 + g2 * g2);
        }
        const float radius = sqrtf(ext2) * p.max_std_dev;
        const double* P = sd.eye[0].proj;
        const float clx = (float)(P[0] * hx + P[4] * hy + P[8] * hz + P[12]);
        const float cly = (float)(P[1] * hx + P[5] * hy + P[9] * hz + P[13]);
        const float clw = (float)(P[3] * hx + P[7] * hy + P[11] * hz + P[15]);
        const float w = fmaxf(clw, 1e-6f);
        const float rx = (float)P[0] * radius / w, ry = (float)P[5] * radius / w;
        const bool inside =
            fabsf(clx / w) - rx <= p.sort_guard + 1.0f && fabsf(cly / w) - ry <= p.sort_guard + 1.0f;
        const bool near_head = -(float)hz <= radius;
        guarded = (float)hz < radius && (inside || near_head);
      }
      const uint32_t kv = key_of_bits(__float_as_uint(__double2float_rn(distance)), sd.sort_bits);
      const bool cull_keys = sd.cull_keys && !sd.keys_only;
      if (!cull_keys && !invisible && guarded) key = kv;
      uint32_t eye_ok = 0;
      if (!sd.keys_only && !invisible) {
#pragma unroll
        for (int v = 0; v < EYES; v++) {
          const DevEye& e = sd.eye[v];
          double ex = hx, ey = hy, ez = hz;
          if (!e.identity) {
            ex = affine_row(e.from_head + 0, hx, hy, hz);
            ey = affine_row(e.from_head + 4, hx, hy, hz);
            ez = affine_row(e.from_head + 8, hx, hy, hz);
          }
          const double* P = e.proj;
          const double clx = dadd(dadd(dadd(dmul(P[0], ex), dmul(P[4], ey)), dmul(P[8], ez)), P[12]);
          const double cly = dadd(dadd(dadd(dmul(P[1], ex), dmul(P[5], ey)), dmul(P[9], ez)), P[13]);
          const double clz = dadd(dadd(dadd(dmul(P[2], ex), dmul(P[6], ey)), dmul(P[10], ez)), P[14]);
          const double clw = dadd(dadd(dadd(dmul(P[3], ex), dmul(P[7], ey)), dmul(P[11], ez)), P[15]);
          // cullDepth and cullClipXY (projection.tsl.ts:132-140)
          const double limit = dmul(fmin((double)p.clip_xy, 2.0), clw);
          const bool culled = ez >= 0.0 || clz < dmul(sd.ndc_z_min, clw) || clz >= clw || fabs(clx) > limit ||
                              fabs(cly) > limit;
          if (!culled) {
            eye_ok |= 1u << v;
            s_eye[v][j] = PerEye{ex, ey, ez, clx, cly, clw};
          }
        }
      }
      candidate = eye_ok != 0;
      s_eye_ok[j] = (uint8_t)eye_ok;
      if (candidate) {
        s_centre[0][j] = cx;
        s_centre[1][j] = cy;
        s_centre[2][j] = cz;
        s_keyval[j] = kv;
      } else if (!sd.keys_only) {
        // culled in every eye: zeros, as a zero opacity byte marks a culled eye
#pragma unroll
        for (int v = 0; v < EYES; v++) {
          const uint64_t ei = (uint64_t)v * sd.out_n + gi;
          if (out.mean2d) reinterpret_cast<float2*>(out.mean2d)[ei] = make_float2(0.f, 0.f);
          if (out.conic) out.conic[ei * 3 + 0] = out.conic[ei * 3 + 1] = out.conic[ei * 3 + 2] = 0.f;
          if (out.depth) out.depth[ei] = 0.f;
          if (out.opacity) out.opacity[ei] = 0.f;
          if (out.rgb) out.rgb[ei * 3 + 0] = out.rgb[ei * 3 + 1] = out.rgb[ei * 3 + 2] = 0.f;
          if (out.radii) out.radii[ei * 3 + 0] = out.radii[ei * 3 + 1] = out.radii[ei * 3 + 2] = 0.f;
          if (out.words) reinterpret_cast<uint4*>(out.words)[gi * EYES + v] = make_uint4(0u, 0u, 0u, 0u);
        }
      }
    }
    s_key[j] = key;
    // compact the candidates, in tile order
    const uint32_t ballot = __ballot_sync(0xffffffffu, candidate);
    if (lane == 0) s_warp_count[warp] = __popc(ballot);
    __syncthreads();
    int before = 0, n_cand = 0;
#pragma unroll
    for (int w = 0; w < kTile / 32; w++) {
      const int c = s_warp_count[w];
      if (w < warp) before += c;
      n_cand += c;
    }
    if (candidate) s_list[before + __popc(ballot & ((1u << lane) - 1u))] = (uint16_t)j;
    __syncthreads();

    // ---- phase 2: the candidates: SH, covariance, ewa (float64) ----
    if (tid < n_cand) {
      const int c = s_list[tid];
      const uint64_t gc = sd.out_offset + i0 + (uint64_t)c;
      float cxf, cyf, czf, opac, ls[3];
      read_centre<LAYOUT, DEG, CDT>(st, c, cxf, cyf, czf, opac, ls);
      double rgb[3];
      const int cap = min(p.max_sh_degree, DEG);
      colour<LAYOUT, DEG, CDT>(st, c, s_centre[0][c] - sd.origin[0], s_centre[1][c] - sd.origin[1],
                               s_centre[2][c] - sd.origin[2], cap, rgb);
      // prepareSplat (float64)
      double op = opac, inflate2 = 1.0;
      if (op > 1.0) {
        op = fmin(op * 4.0 - 3.0, 5.0);
        if (p.lod_inflate) {
          inflate2 = exp((op * op - 1.0) * (2.0 / (3.0 * 2.718281828459045)));
          op = 1.0;
        }
      }
      const float std_dev = op > 1.0 ? (float)((double)p.max_std_dev + (op - 1.0) * 0.7) : p.max_std_dev;
      const double s2x = exp(2.0 * (double)ls[0]) * inflate2;
      const double s2y = exp(2.0 * (double)ls[1]) * inflate2;
      const double s2z = exp(2.0 * (double)ls[2]) * inflate2;
      double q[4];
      read_quat<LAYOUT, DEG, CDT>(st, c, q);
      {
        const double ql2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        if (ql2 > 0.0) {
          const double qi = 1.0 / sqrt(ql2);
          q[0] *= qi;
          q[1] *= qi;
          q[2] *= qi;
          q[3] *= qi;
        } else {
          q[0] = q[1] = q[2] = 0.0;
          q[3] = 1.0;
        }
      }
      const double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
      const double R[9] = {1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy - qw * qz), 2.0 * (qx * qz + qw * qy),
                           2.0 * (qx * qy + qw * qz), 1.0 - 2.0 * (qx * qx + qz * qz), 2.0 * (qy * qz - qw * qx),
                           2.0 * (qx * qz - qw * qy), 2.0 * (qy * qz + qw * qx), 1.0 - 2.0 * (qx * qx + qy * qy)};
      const uint32_t eye_ok = s_eye_ok[c];
      bool any_visible = false;
#pragma unroll
      for (int v = 0; v < EYES; v++) {
        const DevEye& e = sd.eye[v];
        const uint64_t ei = (uint64_t)v * sd.out_n + gc;
        bool ok = (eye_ok >> v) & 1u;
        double ex = 0, ey = 0, ez = -1, clx = 0, cly = 0, clw = 1;
        if (ok) {
          const PerEye pe = s_eye[v][c];
          ex = pe.ex;
          ey = pe.ey;
          ez = pe.ez;
          clx = pe.clx;
          cly = pe.cly;
          clw = pe.clw;
        }
        // depth of field (projection.tsl.ts:117-125)
        float blur = p.blur_amount;
        const float fz = (float)ez;
        if (p.focal_distance > 0.0f && p.aperture_tan > 0.0f && fz < 0.0f) {
          const float depth = -fz;
          const float coc_view = fabsf(depth - p.focal_distance) * p.aperture_tan;
          const float focal_pixels = (float)sd.height * 0.5f * e.proj11;
          const float coc = e.ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
          blur = fminf(fmaxf(coc * coc, blur), p.max_pixel_radius * p.max_pixel_radius);
        }
        double a_d = 0.0, b_d = 0.0, d_d = 0.0, det_d = 1.0, opacity_cd = 0.0;
        float scale1 = 0.f, scale2 = 0.f, angle = 0.f;
        if (ok) {
          // J (projections.tsl.ts:108-118)
          double j1x, j1y, j2x = 0.0, j2y = 0.0;
          if (e.ortho) {
            j1x = e.focal_d[0];
            j1y = e.focal_d[1];
          } else {
            const double inv_z = 1.0 / ez;
            j1x = e.focal_d[0] * inv_z;
            j1y = e.focal_d[1] * inv_z;
            j2x = -(j1x * ex) * inv_z;
            j2y = -(j1y * ey) * inv_z;
          }
          const double* W = e.wd;  // object -> eye 3x3
          const double w0x = j1x * W[0] + j2x * W[6], w0y = j1x * W[1] + j2x * W[7], w0z = j1x * W[2] + j2x * W[8];
          const double w1x = j1y * W[3] + j2y * W[6], w1y = j1y * W[4] + j2y * W[7], w1z = j1y * W[5] + j2y * W[8];
          const double u00 = w0x * R[0] + w0y * R[3] + w0z * R[6];
          const double u01 = w0x * R[1] + w0y * R[4] + w0z * R[7];
          const double u02 = w0x * R[2] + w0y * R[5] + w0z * R[8];
          const double u10 = w1x * R[0] + w1y * R[3] + w1z * R[6];
          const double u11 = w1x * R[1] + w1y * R[4] + w1z * R[7];
          const double u12 = w1x * R[2] + w1y * R[5] + w1z * R[8];
          const double ra = u00 * u00 * s2x + u01 * u01 * s2y + u02 * u02 * s2z;
          const double rd = u10 * u10 * s2x + u11 * u11 * s2y + u12 * u12 * s2z;
          b_d = u00 * u10 * s2x + u01 * u11 * s2y + u02 * u12 * s2z;
          const double m0 = u01 * u12 - u02 * u11;
          const double m1 = u02 * u10 - u00 * u12;
          const double m2 = u00 * u11 - u01 * u10;
          const double det_t = m0 * m0 * (s2y * s2z) + m1 * m1 * (s2x * s2z) + m2 * m2 * (s2x * s2y);
          const double pre = p.pre_blur_amount, full = (double)p.pre_blur_amount + (double)blur;
          const double det_orig = det_t + pre * (ra + rd) + pre * pre;
          det_d = det_t + full * (ra + rd) + full * full;
          a_d = ra + full;
          d_d = rd + full;
          opacity_cd = op * sqrt(fmax(0.0, det_orig / det_d));
          const double contribution = opacity_cd * 6.283185307179586 * sqrt(fmax(0.0, det_d));
          // boundFromCov (projection.tsl.ts:223-240)
          const float a = (float)a_d, b = (float)b_d, d = (float)d_d, det = (float)det_d;
          const float half = (a - d) * 0.5f;
          const float eigen1 = (a + d) * 0.5f + sqrtf(half * half + b * b);
          const float eigen2 = eigen1 > 0.0f ? fmaxf(det / eigen1, 0.0f) : 0.0f;
          scale1 = fminf(p.max_pixel_radius, std_dev * sqrtf(fmaxf(eigen1, 0.0f)));
          scale2 = fminf(p.max_pixel_radius, std_dev * sqrtf(eigen2));
          const bool bound_ok = scale1 >= p.min_pixel_radius || scale2 >= p.min_pixel_radius;
          if (bound_ok) {
            float vx, vy;
            if (fabsf(a - eigen1) >= fabsf(d - eigen1)) {
              vx = b;
              vy = eigen1 - a;
            } else {
              vx = eigen1 - d;
              vy = b;
            }
            const float l2 = vx * vx + vy * vy;
            if (l2 > 0.0f) {
              const float inv = rsqrtf(l2);
              vx *= inv;
              vy *= inv;
            } else {
              vx = 1.0f;
              vy = 0.0f;
            }
            angle = atan2f(vy, vx);
            if (angle < 0.0f) angle += 3.14159265358979f;
          }
          ok = opacity_cd >= (double)p.min_alpha && contribution >= (double)p.min_contribution && bound_ok;
        }
        if (ok) {
          const double inv_w = 1.0 / clw;
          const double ndcx = clx * inv_w, ndcy = cly * inv_w;
          const double inv_det = 1.0 / det_d;
          if (out.mean2d) {
            reinterpret_cast<float2*>(out.mean2d)[ei] =
                make_float2((float)((ndcx + 1.0) * 0.5 * sd.width), (float)((ndcy + 1.0) * 0.5 * sd.height));
          }
          if (out.conic) {
            out.conic[ei * 3 + 0] = (float)(d_d * inv_det);
            out.conic[ei * 3 + 1] = (float)(-b_d * inv_det);
            out.conic[ei * 3 + 2] = (float)(a_d * inv_det);
          }
          if (out.depth) out.depth[ei] = -fz;
          const float opacity_c = (float)opacity_cd;
          if (out.opacity) out.opacity[ei] = opacity_c;
          if (out.rgb) {
            out.rgb[ei * 3 + 0] = (float)rgb[0];
            out.rgb[ei * 3 + 1] = (float)rgb[1];
            out.rgb[ei * 3 + 2] = (float)rgb[2];
          }
          if (out.radii) {
            out.radii[ei * 3 + 0] = scale1;
            out.radii[ei * 3 + 1] = scale2;
            out.radii[ei * 3 + 2] = angle;
          }
          if (out.words) {
            const float stored = opacity_c > 1.0f ? (opacity_c + 3.0f) * 0.25f : opacity_c;
            uint4 wv;
            wv.x = encode_fixed16((float)ndcx) | (encode_fixed16((float)ndcy) << 16);
            wv.y = encode_depth20(fz) | (encode_angle12(angle) << 20);
            wv.z = encode_ext_rgb((float)rgb[0], (float)rgb[1], (float)rgb[2]);
            wv.w = encode_opacity8(stored) | (encode_log_scale12(scale1) << 8) | (encode_log_scale12(scale2) << 20);
            reinterpret_cast<uint4*>(out.words)[gc * EYES + v] = wv;
          }
          any_visible = true;
        } else {
          if (out.mean2d) reinterpret_cast<float2*>(out.mean2d)[ei] = make_float2(0.f, 0.f);
          if (out.conic) out.conic[ei * 3 + 0] = out.conic[ei * 3 + 1] = out.conic[ei * 3 + 2] = 0.f;
          if (out.depth) out.depth[ei] = 0.f;
          if (out.opacity) out.opacity[ei] = 0.f;
          if (out.rgb) out.rgb[ei * 3 + 0] = out.rgb[ei * 3 + 1] = out.rgb[ei * 3 + 2] = 0.f;
          if (out.radii) out.radii[ei * 3 + 0] = out.radii[ei * 3 + 1] = out.radii[ei * 3 + 2] = 0.f;
          if (out.words) reinterpret_cast<uint4*>(out.words)[gc * EYES + v] = make_uint4(0u, 0u, 0u, 0u);
        }
      }
      if (sd.cull_keys && any_visible) s_key[c] = s_keyval[c];
    }
    __syncthreads();

    // ---- keys (coalesced) and their digit histogram ----
    if (live && out.keys) out.keys[gi] = s_key[j];
    if constexpr (HIST) {
      const uint32_t kk = s_key[j];
      const bool valid = live && kk != invalid_key(sd.sort_bits);
      for (int pl = 0; pl < hist.passes; pl++) hist_add(s_hist[pl], (kk >> (8 * pl)) & 0xffu, valid);
      const uint32_t nv = (uint32_t)__popc(__ballot_sync(0xffffffffu, valid));
      if (lane == 0 && nv) atomicAdd(&s_valid, nv);
    }
    __syncthreads();  // stage s is free
    if (tid == 0) {
      const uint32_t tn = t + kStages * stride;
      if (tn < total_tiles) issue(s, tn);
    }
  }
  if constexpr (HIST) {
    __syncthreads();
    if (hist_seg >= 0) {
      for (int w = tid; w < hist.passes * kRadix; w += kTile) {
        const uint32_t c = (&s_hist[0][0])[w];
        if (c) atomicAdd(&hist.hist[(size_t)hist_seg * hist.passes * kRadix + w], c);
      }
      if (tid == 0 && s_valid) atomicAdd(&hist.valid[hist_seg], s_valid);
    }
  }
}

using ProjKernel = void (*)(const ProjDesc*, int, uint32_t, ProjOutputs, ProjHist, uint32_t*);

struct Picked {
  ProjKernel fn;
  int smem;
};

template <int LAYOUT, int DEG, int CDT, int EYES, bool HIST>
Picked picked() {
  return {k_project<LAYOUT, DEG, CDT, EYES, HIST>, kStages * Stage<LAYOUT, DEG, CDT>::kBytes};
}

template <int LAYOUT, int DEG, int CDT>
Picked pick_eyes(int eyes, bool hist) {
  if (eyes == 2) return hist ? picked<LAYOUT, DEG, CDT, 2, true>() : picked<LAYOUT, DEG, CDT, 2, false>();
  return hist ? picked<LAYOUT, DEG, CDT, 1, true>() : picked<LAYOUT, DEG, CDT, 1, false>();
}

template <int LAYOUT, int CDT>
Picked pick_degree(int degree, int eyes, bool hist) {
  switch (degree) {
    case 0: return pick_eyes<LAYOUT, 0, CDT>(eyes, hist);
    case 1: return pick_eyes<LAYOUT, 1, CDT>(eyes, hist);
    case 2: return pick_eyes<LAYOUT, 2, CDT>(eyes, hist);
    case 3: return pick_eyes<LAYOUT, 3, CDT>(eyes, hist);
    default: return pick_eyes<LAYOUT, 4, CDT>(eyes, hist);
  }
}

Picked pick_kernel(int layout, int degree, int cdt, int eyes, bool hist) {
  if (layout == RDX_LAYOUT_EXT) return pick_degree<RDX_LAYOUT_EXT, RDX_DTYPE_F32>(degree, eyes, hist);
  if (cdt == RDX_DTYPE_F16) return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F16>(degree, eyes, hist);
  return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F32>(degree, eyes, hist);
}

}  // namespace

cudaError_t launch_project(const ProjDesc* descs_dev, const ProjDesc* descs_host, int n_desc, uint32_t total_tiles,
                           const ProjOutputs& out, const ProjHist& hist, uint32_t* error_flag, cudaStream_t stream) {
  if (total_tiles == 0 || n_desc == 0) return cudaSuccess;
  // One kernel per launch: the caller groups objects by table kind
  const ProjDesc& d0 = descs_host[0];
  const Picked k =
      pick_kernel(d0.table.layout, d0.table.sh_degree, d0.table.color_dtype, d0.eyes, hist.hist != nullptr);
  cudaError_t err = cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
  if (err != cudaSuccess) return err;
  int device = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, kTile, k.smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) per_sm = 1;
  const uint32_t grid = min(total_tiles, (uint32_t)(sms * per_sm));
  k.fn<<<grid, kTile, k.smem, stream>>>(descs_dev, n_desc, total_tiles, out, hist, error_flag);
  return cudaGetLastError();
}

}  // namespace rdx
