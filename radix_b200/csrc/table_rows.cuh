// Row access of the splat tables for the projection kernels: the SH basis,
// the columns of raw / ext / cov / packed rows, and the base colour plus SH of
// a row (src/gpu/splats.tsl.ts:63-71, 104-154; src/gpu/sh.tsl.ts:32-139,
// 219-266; src/core/splats.ts:10-32, 223-306; src/core/sh.ts:13-24, 114-174).
// Shared by the ewa projection (project.cu) and the ray methods (rays.cu).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {
namespace {

template <int DEG>
struct ShCount {
  static constexpr int value = DEG == 0 ? 0 : (DEG == 1 ? 3 : (DEG == 2 ? 8 : (DEG == 3 ? 15 : 24)));
};

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

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// The template parameter VAR is the raw layout's colour type (RDX_DTYPE_*),
// and the SH codec (RDX_SH_*) of the other layouts.

// Phase 1's fields of row i: centre, opacity, ln scales in float64 (-inf: a
// zero scale). `zero` is set when the splat's covariance is zero (every
// scale, or every variance, underflows to 0): cullInvisible's zero cov.
template <int LAYOUT>
__device__ __forceinline__ void load_head(const DevTable& t, uint64_t i, float c[3], float& opacity, double ls[3],
                                          bool& zero) {
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    const float* cp = t.centers + i * 3;
    const float* lp = t.log_scales + i * 3;
    c[0] = __ldg(cp);
    c[1] = __ldg(cp + 1);
    c[2] = __ldg(cp + 2);
    ls[0] = __ldg(lp);
    ls[1] = __ldg(lp + 1);
    ls[2] = __ldg(lp + 2);
    opacity = __ldg(t.opacities + i);
  } else if constexpr (LAYOUT == RDX_LAYOUT_PACKED) {
    // packedCodec.decode (src/core/splats.ts:288-306), src/gpu/splats.tsl.ts:141-154
    const uint4 P = __ldg(reinterpret_cast<const uint4*>(t.packed) + i);
    c[0] = half_bits_to_float(P.y);
    c[1] = half_bits_to_float(P.y >> 16);
    c[2] = half_bits_to_float(P.z);
    opacity = (float)(P.x >> 24) * (1.0f / 255.0f);
    const double lmin = t.packed_encoding[2];
    const double step = ((double)t.packed_encoding[3] - lmin) / 254.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const uint32_t code = (P.w >> (8 * k)) & 0xffu;
      ls[k] = code == 0u ? -INFINITY : lmin + (double)(code - 1u) * step;
    }
  } else {
    // extA / covA and extB / covB (src/core/splats.ts:10-32; src/gpu/splats.tsl.ts:63-71, 104-118)
    const uint4 A = __ldg(reinterpret_cast<const uint4*>(t.ext_a) + i);
    const uint4 B = __ldg(reinterpret_cast<const uint4*>(t.ext_b) + i);
    c[0] = __uint_as_float(A.x);
    c[1] = __uint_as_float(A.y);
    c[2] = __uint_as_float(A.z);
    opacity = (float)(A.w >> 24) * (1.0f / 128.0f);
    // ext: ln scales; cov: ln variances (the same half fields)
    ls[0] = half_bits_to_float(B.y);
    ls[1] = half_bits_to_float(B.y >> 16);
    ls[2] = half_bits_to_float(B.z);
  }
  if constexpr (LAYOUT == RDX_LAYOUT_COV) {
    zero = ls[0] == -INFINITY && ls[1] == -INFINITY && ls[2] == -INFINITY;  // exp(-inf) variances
  } else {
    // exp(2 ln s) underflows to 0 below ln s = -372.6
    zero = ls[0] < -372.6 && ls[1] < -372.6 && ls[2] < -372.6;
  }
}

// Phase 1's columns of the chunk starting at row j0 into L2 (a 128-byte line per lane)
template <int LAYOUT>
__device__ __forceinline__ void prefetch_head(const DevTable& t, uint64_t j0, uint64_t count, int lane) {
  const unsigned char* base;
  uint64_t off, size;
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    // centres and ln scales: 384 bytes each (3 lines), opacities 128 bytes (1 line)
    if (lane < 3) {
      base = reinterpret_cast<const unsigned char*>(t.centers);
      off = j0 * 12 + (uint64_t)lane * 128;
      size = count * 12;
    } else if (lane < 6) {
      base = reinterpret_cast<const unsigned char*>(t.log_scales);
      off = j0 * 12 + (uint64_t)(lane - 3) * 128;
      size = count * 12;
    } else if (lane < 7) {
      base = reinterpret_cast<const unsigned char*>(t.opacities);
      off = j0 * 4;
      size = count * 4;
    } else {
      return;
    }
  } else if constexpr (LAYOUT == RDX_LAYOUT_PACKED) {
    if (lane >= 4) return;  // 512 bytes
    base = reinterpret_cast<const unsigned char*>(t.packed);
    off = j0 * 16 + (uint64_t)lane * 128;
    size = count * 16;
  } else {
    // A and B: 512 bytes each (4 lines)
    if (lane >= 8) return;
    base = reinterpret_cast<const unsigned char*>(lane < 4 ? t.ext_a : t.ext_b);
    off = j0 * 16 + (uint64_t)(lane & 3) * 128;
    size = count * 16;
  }
  if (off < size) prefetch_l2(base + off);
}

template <int DEG, int VAR>
struct ColorRow {
  static constexpr int kValues = (1 + ShCount<DEG>::value) * 3;
  static constexpr int kBytes = kValues * (VAR == RDX_DTYPE_F16 ? 2 : 4);
  static constexpr int kVec = kBytes % 16 == 0 ? 16 : (kBytes % 8 == 0 ? 8 : (kBytes % 4 == 0 ? 4 : 2));
};

// Texels of an SH entry in codec VAR: ext one word per coefficient, packed
// 10 / 26 / 48 / 76 bytes for degree 1 / 2 / 3 / 4 (src/core/sh.ts:13-24)
template <int DEG, int VAR>
struct ShTexels {
  static constexpr int value = VAR == RDX_SH_PACKED ? (DEG == 0 ? 0 : (DEG == 1 ? 1 : (DEG == 2 ? 2 : (DEG == 3 ? 3 : 5))))
                                                    : (ShCount<DEG>::value + 3) / 4;
};

// Texel k of splat i's SH entry: its per-splat channel, or its palette entry
// (sh.tsl.ts:219-233; a label past the palette reads the last entry)
__device__ __forceinline__ const uint4* sh_texel(const DevTable& t, uint64_t i, int k) {
  if (t.sh_palette) {
    uint64_t label = __ldg(t.sh_label + i);
    if (label >= t.sh_palette_size) label = t.sh_palette_size - 1;
    return reinterpret_cast<const uint4*>(t.sh_palette) + label * t.sh_stride + (uint64_t)k;
  }
  return reinterpret_cast<const uint4*>(t.ext_sh[k]) + i;
}

// Phase 2's rows of a queued splat into L2 while the queue fills
template <int LAYOUT, int DEG, int VAR>
__device__ __forceinline__ void prefetch_rows(const DevTable& t, uint64_t i) {
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    prefetch_l2(t.quats + i * 4);
    const unsigned char* row = reinterpret_cast<const unsigned char*>(t.colors) + i * ColorRow<DEG, VAR>::kBytes;
#pragma unroll
    for (int off = 0; off < ColorRow<DEG, VAR>::kBytes; off += 128) prefetch_l2(row + off);
    prefetch_l2(row + ColorRow<DEG, VAR>::kBytes - 1);
  } else {
#pragma unroll
    for (int k = 0; k < ShTexels<DEG, VAR>::value; k++) prefetch_l2(sh_texel(t, i, k));
  }
}

template <int LAYOUT>
__device__ __forceinline__ void load_quat(const DevTable& t, uint64_t i, double q[4]) {
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(t.quats) + i);
    q[0] = v.x;
    q[1] = v.y;
    q[2] = v.z;
    q[3] = v.w;
  } else if constexpr (LAYOUT == RDX_LAYOUT_PACKED) {
    const uint4 P = __ldg(reinterpret_cast<const uint4*>(t.packed) + i);
    decode_quat_oct_f64<8, 8>((P.z >> 16) | ((P.w >> 24) << 16), q);
  } else if constexpr (LAYOUT == RDX_LAYOUT_EXT) {
    decode_quat_oct32_f64(__ldg(reinterpret_cast<const uint4*>(t.ext_b) + i).w, q);
  } else {
    q[0] = q[1] = q[2] = 0.0;  // the cov layout stores no rotation
    q[3] = 1.0;
  }
}

// covB's object-space covariance: xx, yy, zz, xy, xz, yz (src/core/splats.ts:223-266)
__device__ __forceinline__ double decode_correlation(double e) {
  return e == 0.0 ? 0.0 : (e > 0.0 ? -1.0 : 1.0) * exp(-fabs(e));
}

__device__ __forceinline__ void load_cov(const DevTable& t, uint64_t i, double cov[6]) {
  const uint4 B = __ldg(reinterpret_cast<const uint4*>(t.ext_b) + i);
  const double xx = exp((double)half_bits_to_float(B.y)), yy = exp((double)half_bits_to_float(B.y >> 16)),
               zz = exp((double)half_bits_to_float(B.z));
  cov[0] = xx;
  cov[1] = yy;
  cov[2] = zz;
  cov[3] = decode_correlation(half_bits_to_float(B.z >> 16)) * sqrt(xx * yy);
  cov[4] = decode_correlation(half_bits_to_float(B.w)) * sqrt(xx * zz);
  cov[5] = decode_correlation(half_bits_to_float(B.w >> 16)) * sqrt(yy * zz);
}

template <int BYTES>
__device__ __forceinline__ void load_vec(const unsigned char* p, unsigned char* dst) {
  if constexpr (BYTES == 16) {
    *reinterpret_cast<uint4*>(dst) = __ldg(reinterpret_cast<const uint4*>(p));
  } else if constexpr (BYTES == 8) {
    *reinterpret_cast<uint2*>(dst) = __ldg(reinterpret_cast<const uint2*>(p));
  } else if constexpr (BYTES == 4) {
    *reinterpret_cast<uint32_t*>(dst) = __ldg(reinterpret_cast<const unsigned int*>(p));
  } else {
    *reinterpret_cast<unsigned short*>(dst) = __ldg(reinterpret_cast<const unsigned short*>(p));
  }
}

// Base rgb + SH (float64) of row i seen along (dx, dy, dz), clamped at 0 when
// the table has SH (GpuShReader.apply); without SH no clamp
template <int LAYOUT, int DEG, int VAR>
__device__ __forceinline__ void colour(const DevTable& t, uint64_t i, double dx, double dy, double dz, int cap,
                                       double rgb[3], const uint4* staged = nullptr) {
  constexpr int K = ShCount<DEG>::value;
  double acc[3] = {0.0, 0.0, 0.0};
  const double l2 = dx * dx + dy * dy + dz * dz;
  const double inv = l2 > 0.0 ? 1.0 / sqrt(l2) : 0.0;
  const double x = dx * inv, y = dy * inv, z = dz * inv;
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    using CR = ColorRow<DEG, VAR>;
    alignas(16) unsigned char buf[(CR::kBytes + 15) / 16 * 16];
    if constexpr (CR::kBytes % 16 == 0) {
      if (staged) {  // the row a warp staged in shared memory
#pragma unroll
        for (int b = 0; b < CR::kBytes / 16; b++) reinterpret_cast<uint4*>(buf)[b] = staged[b];
      }
    }
    if (!staged) {
      const unsigned char* row = reinterpret_cast<const unsigned char*>(t.colors) + i * CR::kBytes;
#pragma unroll
      for (int b = 0; b < CR::kBytes; b += CR::kVec) load_vec<CR::kVec>(row + b, buf + b);
    }
    auto value = [&](int v) -> double {
      if constexpr (VAR == RDX_DTYPE_F16) {
        return (double)__half2float(*reinterpret_cast<const __half*>(buf + v * 2));
      } else {
        return (double)*reinterpret_cast<const float*>(buf + v * 4);
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
    if constexpr (LAYOUT == RDX_LAYOUT_PACKED) {
      // rgbMin + byte / 255 * (rgbMax - rgbMin)
      const uint32_t w = __ldg(reinterpret_cast<const uint4*>(t.packed) + i).x;
      const double rmin = t.packed_encoding[0], range = (double)t.packed_encoding[1] - rmin;
#pragma unroll
      for (int c = 0; c < 3; c++) rgb[c] = rmin + ((double)((w >> (8 * c)) & 0xffu) / 255.0) * range;
    } else {
      decode_ext_rgb_f64(__ldg(reinterpret_cast<const uint4*>(t.ext_b) + i).x, rgb);
    }
    if constexpr (K > 0) {
      constexpr int kTexels = ShTexels<DEG, VAR>::value;
      uint32_t words[kTexels * 4];
#pragma unroll
      for (int k = 0; k < kTexels; k++) {
        const uint4 T = __ldg(sh_texel(t, i, k));
        words[k * 4 + 0] = T.x;
        words[k * 4 + 1] = T.y;
        words[k * 4 + 2] = T.z;
        words[k * 4 + 3] = T.w;
      }
      auto byte_at = [&](int b) -> uint32_t { return (words[b >> 2] >> ((b & 3) * 8)) & 0xffu; };
#pragma unroll
      for (int band = 1; band <= DEG; band++) {
        if (band <= cap) {
          double basis[9];
          const int nb = sh_basis_band(band, x, y, z, basis);
          // packed: the band's scale byte, then its sint8 values (sh.ts:156-168)
          constexpr int kStart[5] = {0, 0, 10, 26, 48};
          double scale = 0.0;
          if constexpr (VAR == RDX_SH_PACKED) {
            const uint32_t code = byte_at(kStart[band]);
            scale = code == 0u ? 0.0 : exp2(((double)code - 192.0) / 16.0) / 127.0;
          }
#pragma unroll
          for (int k = 0; k < 9; k++) {
            if (k < nb) {
              double c[3];
              if constexpr (VAR == RDX_SH_PACKED) {
#pragma unroll
                for (int ch = 0; ch < 3; ch++) {
                  const int b = kStart[band] + 1 + k * 3 + ch;
                  c[ch] = (double)(int)(signed char)byte_at(b) * scale;
                }
              } else {
                decode_ext_rgb_f64(words[band * band - 1 + k], c);
              }
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

}  // namespace
}  // namespace rdx
