// Device helpers shared by the kernels: sort keys, Radix's scalar codecs, and
// the word encoders of the ewa projection.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

namespace rdx {

// The bytes [src, src + len) into words of shared memory (dst[j] holds bytes
// 4j to 4j + 3), copied by one warp with aligned word loads, funnel-shifted
// pairs of them when src is off a word boundary; every word read holds at
// least one of the bytes. kBatch loads a lane are in flight before their stores.
__device__ __forceinline__ void warp_copy_bytes(const unsigned char* src, uint32_t len, uint32_t* dst, uint32_t lane) {
  constexpr uint32_t kBatch = 16;
  const uint32_t shift = (uint32_t)((uintptr_t)src & 3u);
  const uint32_t* aw = reinterpret_cast<const uint32_t*>(src - shift);
  const uint32_t n_out = (len + 3) / 4, n_in = (len + shift + 3) / 4;
  for (uint32_t j0 = lane; j0 < n_out; j0 += 32 * kBatch) {
    uint32_t lo[kBatch], hi[kBatch];
#pragma unroll
    for (uint32_t b = 0; b < kBatch; b++) {
      const uint32_t j = j0 + 32 * b;
      lo[b] = j < n_out ? __ldg(aw + j) : 0u;
      hi[b] = shift != 0 && j + 1 < n_in ? __ldg(aw + j + 1) : 0u;
    }
#pragma unroll
    for (uint32_t b = 0; b < kBatch; b++) {
      const uint32_t j = j0 + 32 * b;
      if (j < n_out) dst[j] = shift == 0 ? lo[b] : __funnelshift_r(lo[b], hi[b], 8 * shift);
    }
  }
}

// Non-contracted float64 arithmetic: the sort-key distance and the centre
// culls round exactly as the float64 CPU oracle does.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

// Row r of a 3x4 (or 4x4) transform applied to (x, y, z, 1): ((m0 x + m1 y) + m2 z) + m3
__device__ __forceinline__ double affine_row(const double* m, double x, double y, double z) {
  return dadd(dadd(dadd(dmul(m[0], x), dmul(m[1], y)), dmul(m[2], z)), m[3]);
}

// Key of the float32 bits of a distance (src/core/sort.ts:46-58)
__device__ __forceinline__ uint32_t key_of_bits(uint32_t f, int bits) {
  const uint32_t mask = bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
  if (!(f < 0x7f800000u)) return mask;
  uint32_t q;
  if (bits == 32) {
    q = f;
  } else if (bits == 24) {
    q = f >> 7;
  } else {
    const uint32_t lo = 95u << 23, hi = (159u << 23) - 1u;
    q = (min(max(f, lo), hi) - lo) >> 13;
  }
  const uint32_t valid_max = (0xffu << (bits - 8)) - 1u;
  return min(mask ^ q, valid_max);
}

__device__ __forceinline__ uint32_t invalid_key(int bits) {
  return bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
}

// Ext rgb word (src/core/encoding.ts:233-239, src/gpu/encoding.tsl.ts:35-44):
// 8-bit magnitudes times 2^(e - 15) / 255, 3 sign bits
__device__ __forceinline__ float3 decode_ext_rgb(uint32_t w) {
  const float unit = __uint_as_float((((w >> 27) & 0x1fu) + 112u) << 23);
  float r = (float)(w & 0xffu) * unit * (1.0f / 255.0f);
  float g = (float)((w >> 8) & 0xffu) * unit * (1.0f / 255.0f);
  float b = (float)((w >> 16) & 0xffu) * unit * (1.0f / 255.0f);
  if (w & 0x1000000u) r = -r;
  if (w & 0x2000000u) g = -g;
  if (w & 0x4000000u) b = -b;
  return make_float3(r, g, b);
}

// The same word decoded exactly in float64 (m * 2^(e - 15) / 255)
__device__ __forceinline__ void decode_ext_rgb_f64(uint32_t w, double* out) {
  const double unit = __longlong_as_double((long long)((((w >> 27) & 0x1fu) + 1008u)) << 52) / 255.0;
  out[0] = (double)(w & 0xffu) * unit * ((w & 0x1000000u) ? -1.0 : 1.0);
  out[1] = (double)((w >> 8) & 0xffu) * unit * ((w & 0x2000000u) ? -1.0 : 1.0);
  out[2] = (double)((w >> 16) & 0xffu) * unit * ((w & 0x4000000u) ? -1.0 : 1.0);
}

__device__ __forceinline__ float half_bits_to_float(uint32_t h) {
  return __half2float(__ushort_as_half((unsigned short)(h & 0xffffu)));
}

// QuatOct32 (src/core/encoding.ts:101-110, src/gpu/encoding.tsl.ts:113-118):
// octahedral axis 10 + 10 bits, angle 0..pi in 12 bits; code 0 axis -> zero
__device__ __forceinline__ float4 decode_quat_oct32(uint32_t code) {
  const uint32_t axis = code & 0xfffffu;
  float x = 0.f, y = 0.f, z = 0.f;
  if (axis != 0u) {
    x = (float)(axis & 1023u) * (2.0f / 1023.0f) - 1.0f;
    y = (float)((axis >> 10) & 1023u) * (2.0f / 1023.0f) - 1.0f;
    z = 1.0f - fabsf(x) - fabsf(y);
    const float t = fmaxf(-z, 0.0f);
    x += x >= 0.0f ? -t : t;
    y += y >= 0.0f ? -t : t;
    const float inv = rsqrtf(x * x + y * y + z * z);
    x *= inv;
    y *= inv;
    z *= inv;
  }
  const float half_angle = (float)((code >> 20) & 4095u) * (1.5707963267948966f / 4095.0f);
  float s, c;
  sincosf(half_angle, &s, &c);
  return make_float4(x * s, y * s, z * s, c);
}

// A quaternion code in float64 (the oracle's precision): an octahedral axis
// of AXIS + AXIS bits, then the angle 0..pi in ANGLE bits
// (src/core/encoding.ts:49-67, 101-110; QuatOct32 = 10 + 10 + 12, QuatOct24 = 8 + 8 + 8)
template <int AXIS, int ANGLE>
__device__ __forceinline__ void decode_quat_oct_f64(uint32_t code, double q[4]) {
  constexpr uint32_t kMax = (1u << AXIS) - 1u;
  constexpr uint32_t kAngleMax = (1u << ANGLE) - 1u;
  const uint32_t axis = code & ((1u << (2 * AXIS)) - 1u);
  double x = 0.0, y = 0.0, z = 0.0;
  if (axis != 0u) {
    x = (double)(axis & kMax) / (double)kMax * 2.0 - 1.0;
    y = (double)((axis >> AXIS) & kMax) / (double)kMax * 2.0 - 1.0;
    z = 1.0 - fabs(x) - fabs(y);
    const double t = fmax(-z, 0.0);
    x += x >= 0.0 ? -t : t;
    y += y >= 0.0 ? -t : t;
    const double len = sqrt(x * x + y * y + z * z);
    x /= len;
    y /= len;
    z /= len;
  }
  const double angle = (double)((code >> (2 * AXIS)) & kAngleMax) / (double)kAngleMax * 3.14159265358979323846;
  double s, c;
  sincos(angle / 2.0, &s, &c);
  q[0] = x * s;
  q[1] = y * s;
  q[2] = z * s;
  q[3] = c;
}

__device__ __forceinline__ void decode_quat_oct32_f64(uint32_t code, double q[4]) { decode_quat_oct_f64<10, 12>(code, q); }

// ---- the ewa words (src/render/projection.tsl.ts:277-311) ----

__device__ __forceinline__ uint32_t encode_fixed16(float v) {
  return (uint32_t)fminf(fmaxf(floorf((v + 2.0f) * 0.25f * 65535.0f + 0.5f), 0.0f), 65535.0f);
}

__device__ __forceinline__ uint32_t encode_depth20(float view_z) {
  const uint32_t lo = 113u << 23, hi = (145u << 23) - 1u;
  const uint32_t f = min(max(__float_as_uint(-view_z), lo), hi);
  return min((f - lo + 128u) >> 8, 0xfffffu);
}

__device__ __forceinline__ uint32_t encode_angle12(float angle) {
  return (uint32_t)floorf(angle * (4096.0f / 3.14159265358979f) + 0.5f) & 0xfffu;
}

__device__ __forceinline__ uint32_t encode_log_scale12(float scale) {
  const float top = 4094.0f;
  const float l = fminf(fmaxf(log2f(fmaxf(scale, 1e-20f)), -4.0f), 12.0f);
  const float normalized = (l + 4.0f) * (1.0f / 16.0f) * top;
  return (uint32_t)fminf(fmaxf(floorf(normalized + 0.5f), 0.0f), top) + 1u;
}

__device__ __forceinline__ uint32_t encode_opacity8(float opacity) {
  const uint32_t v = (uint32_t)floorf(fminf(fmaxf(opacity * 128.0f, 0.0f), 255.0f) + 0.5f);
  return max(v, 1u);
}

// src/gpu/encoding.tsl.ts:19-33
__device__ __forceinline__ uint32_t encode_ext_rgb(float r, float g, float b) {
  const float m = fmaxf(fabsf(r), fmaxf(fabsf(g), fabsf(b)));
  int base = (m > 0.0f ? (int)ceilf(log2f(m)) : 0) + 15;
  base = min(max(base, 0), 31);
  const float scale = __uint_as_float((uint32_t)(142 - base) << 23) * 255.0f;
  const uint32_t mr = (uint32_t)fminf(floorf(fabsf(r) * scale + 0.5f), 255.0f);
  const uint32_t mg = (uint32_t)fminf(floorf(fabsf(g) * scale + 0.5f), 255.0f);
  const uint32_t mb = (uint32_t)fminf(floorf(fabsf(b) * scale + 0.5f), 255.0f);
  const uint32_t signs = (r < 0.0f ? 1u : 0u) | (g < 0.0f ? 2u : 0u) | (b < 0.0f ? 4u : 0u);
  return mr | (mg << 8) | (mb << 16) | ((((uint32_t)base << 3) | signs) << 24);
}

}  // namespace rdx
