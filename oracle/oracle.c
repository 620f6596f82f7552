/*
 * oracle.c - CPU FP64 restatement of the @sparkjsdev/radix per-frame splat path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker the CUDA kernels are
 * compared against (tests/, the smoke check and the CPU baseline of bench.py);
 * the product never links it. Paths in citations are inside the radix project.
 *
 * Precision: every value is float64, as the reference's CPU functions (JS
 * numbers) are. Where the reference's CPU path rounds to float32 (the
 * distance of a sort key goes through a Float32Array), this does too.
 * Compile with -ffp-contract=off: the sort-key distance and the
 * centre culls must round exactly as the device's non-contracted float64
 * arithmetic does.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.14159265358979323846;
static const double E_CONST = 2.71828182845904523536;

/* ---- sort keys: src/core/sort.ts:29-58 ---- */

#define KEY16_LO (95u << 23)
#define KEY16_HI ((159u << 23) - 1u)
#define FLOAT_BITS_INFINITY 0x7f800000u

uint32_t orc_invalid_key(int bits) { /* sort.ts:37-39 */
  return bits == 32 ? 0xffffffffu : ((1u << bits) - 1u);
}

uint32_t orc_valid_max(int bits) { /* sort.ts:41-43 */
  return (0xffu << (bits - 8)) - 1u;
}

static uint32_t key_of_bits(uint32_t f, int bits) {
  const uint32_t mask = orc_invalid_key(bits);
  if (!(f < FLOAT_BITS_INFINITY)) {
    return mask;
  }
  uint32_t q;
  if (bits == 32) {
    q = f;
  } else if (bits == 24) {
    q = f >> 7;
  } else {
    uint32_t c = f < KEY16_LO ? KEY16_LO : (f > KEY16_HI ? KEY16_HI : f);
    q = (c - KEY16_LO) >> 13;
  }
  uint32_t k = mask ^ q;
  uint32_t vmax = orc_valid_max(bits);
  return k < vmax ? k : vmax;
}

/* SortKeys.compute, sort.ts:46-58: the distance through a Float32Array */
uint32_t orc_sort_key(double distance, int bits) {
  float f32 = (float)distance;
  uint32_t f;
  memcpy(&f, &f32, 4);
  return key_of_bits(f, bits);
}

/* GpuSortKeys.compute, sortKey.tsl.ts:17-26: float32 distance, max(d, 0) */
uint32_t orc_sort_key_f32(float distance, int bits) {
  float d = distance;
  if (!(d > 0.0f) && !isnan(d)) {
    d = 0.0f;
  }
  uint32_t f;
  memcpy(&f, &d, 4);
  return key_of_bits(f, bits);
}

void orc_sort_keys(const double* distances, uint64_t n, int bits, uint32_t* keys) {
  for (uint64_t i = 0; i < n; i++) {
    keys[i] = orc_sort_key(distances[i], bits);
  }
}

/* ---- SortKeys.sort: sort.ts:64-163, the same digit layouts ---- */

static uint32_t hist_lo[65536];
static uint32_t hist_hi[65536];

static void prefix_sum(uint32_t* h, uint32_t last) { /* sort.ts:85-92 */
  uint32_t sum = 0;
  for (uint32_t d = 0; d <= last; d++) {
    uint32_t n = h[d];
    h[d] = sum;
    sum += n;
  }
}

int orc_sort(const uint32_t* keys, uint64_t count, int bits, uint32_t* ordering,
             uint64_t ordering_len, uint32_t* visible_out) {
  if (ordering_len < count) {
    return -1; /* sort.ts:70-72 */
  }
  uint32_t visible = 0;
  if (bits == 16) { /* sort1x16, sort.ts:97-110 */
    memset(hist_lo, 0, sizeof(hist_lo));
    for (uint64_t i = 0; i < count; i++) hist_lo[keys[i] & 0xffffu] += 1;
    visible = (uint32_t)count - hist_lo[0xffff];
    prefix_sum(hist_lo, 0xffff);
    for (uint64_t i = 0; i < count; i++) ordering[hist_lo[keys[i] & 0xffffu]++] = (uint32_t)i;
  } else {
    /* sort11x13 (sort.ts:113-137) and sort2x16 (139-163); 24-bit keys use their low 24 bits */
    const int lo_bits = bits == 24 ? 11 : 16;
    const uint32_t lo_mask = (1u << lo_bits) - 1u;
    const uint32_t hi_last = bits == 24 ? 0x1fffu : 0xffffu;
    const uint32_t key_mask = bits == 24 ? 0xffffffu : 0xffffffffu;
    uint32_t* scratch_index = (uint32_t*)malloc(count ? count * 4 : 4);
    uint16_t* scratch_digit = (uint16_t*)malloc(count ? count * 2 : 2);
    memset(hist_lo, 0, (size_t)(lo_mask + 1) * 4);
    memset(hist_hi, 0, (size_t)(hi_last + 1) * 4);
    for (uint64_t i = 0; i < count; i++) {
      uint32_t k = keys[i] & key_mask;
      hist_lo[k & lo_mask] += 1;
      hist_hi[k >> lo_bits] += 1;
    }
    visible = (uint32_t)count - hist_hi[hi_last];
    prefix_sum(hist_lo, lo_mask);
    prefix_sum(hist_hi, hi_last);
    for (uint64_t i = 0; i < count; i++) {
      uint32_t k = keys[i] & key_mask;
      uint32_t pos = hist_lo[k & lo_mask]++;
      scratch_index[pos] = (uint32_t)i;
      scratch_digit[pos] = (uint16_t)(k >> lo_bits);
    }
    for (uint64_t j = 0; j < count; j++) {
      ordering[hist_hi[scratch_digit[j]]++] = scratch_index[j];
    }
    free(scratch_index);
    free(scratch_digit);
  }
  if (visible_out) *visible_out = visible;
  return 0;
}

/* ---- codecs: src/core/encoding.ts ---- */

double orc_decode_half(uint32_t h) { /* encoding.ts:191-202 */
  double sign = (h & 0x8000u) ? -1.0 : 1.0;
  int exponent = (int)((h >> 10) & 0x1fu);
  double mantissa = (double)(h & 0x3ffu);
  if (exponent == 0) return sign * mantissa * ldexp(1.0, -24);
  if (exponent == 0x1f) return mantissa != 0.0 ? NAN : sign * INFINITY;
  return sign * (1.0 + mantissa / 1024.0) * ldexp(1.0, exponent - 15);
}

/* encoding.ts:156-159 with Float16Array: float64 to half, ties to even */
uint32_t orc_encode_half(double f) {
  uint32_t sign = signbit(f) ? 0x8000u : 0u;
  double a = fabs(f);
  if (isnan(f)) return sign | 0x7e00u;
  if (a >= 65520.0) return sign | 0x7c00u; /* rounds to infinity */
  if (a < ldexp(1.0, -14)) { /* subnormal: multiples of 2^-24 */
    double m = a * ldexp(1.0, 24);
    double r = nearbyint(m); /* ties to even (default rounding mode) */
    return sign | (uint32_t)r;
  }
  int e;
  double frac = frexp(a, &e); /* a = frac * 2^e, frac in [0.5, 1) */
  double m = (frac * 2.0 - 1.0) * 1024.0;
  double r = nearbyint(m);
  int exponent = e - 1 + 15;
  if (r >= 1024.0) {
    r = 0.0;
    exponent += 1;
  }
  if (exponent >= 31) return sign | 0x7c00u;
  return sign | ((uint32_t)exponent << 10) | (uint32_t)r;
}

void orc_decode_ext_rgb(uint32_t w, double rgb[3]) { /* encoding.ts:233-239 */
  double unit = ldexp(1.0, (int)((w >> 27) & 0x1fu) - 15) / 255.0;
  rgb[0] = (double)(w & 0xffu) * unit * ((w & 0x1000000u) ? -1.0 : 1.0);
  rgb[1] = (double)((w >> 8) & 0xffu) * unit * ((w & 0x2000000u) ? -1.0 : 1.0);
  rgb[2] = (double)((w >> 16) & 0xffu) * unit * ((w & 0x4000000u) ? -1.0 : 1.0);
}

static double js_round(double x) { return floor(x + 0.5); } /* Math.round */

uint32_t orc_encode_ext_rgb(const double rgb[3]) { /* encoding.ts:219-231 */
  double max_abs = fmax(fabs(rgb[0]), fmax(fabs(rgb[1]), fabs(rgb[2])));
  int base = (max_abs > 0 ? (int)ceil(log2(max_abs)) : 0) + 15;
  base = base < 0 ? 0 : (base > 31 ? 31 : base);
  double scale = 255.0 * ldexp(1.0, 15 - base);
  uint32_t m[3];
  for (int c = 0; c < 3; c++) {
    double v = js_round(fabs(rgb[c]) * scale);
    m[c] = (uint32_t)(v > 255.0 ? 255.0 : v);
  }
  uint32_t signs = (rgb[0] < 0 ? 1u : 0u) | (rgb[1] < 0 ? 2u : 0u) | (rgb[2] < 0 ? 4u : 0u);
  return m[0] | (m[1] << 8) | (m[2] << 16) | ((((uint32_t)base << 3) | signs) << 24);
}

void orc_decode_oct(uint32_t code, int bits, double out[3]) { /* encoding.ts:49-67 */
  if (code == 0) {
    out[0] = out[1] = out[2] = 0.0;
    return;
  }
  double max = (double)((1u << bits) - 1u);
  uint32_t mask = (1u << bits) - 1u;
  double x = (double)(code & mask) / max * 2.0 - 1.0;
  double y = (double)((code >> bits) & mask) / max * 2.0 - 1.0;
  double z = 1.0 - fabs(x) - fabs(y);
  double t = fmax(-z, 0.0);
  x += x >= 0 ? -t : t;
  y += y >= 0 ? -t : t;
  double len = sqrt(x * x + y * y + z * z);
  out[0] = x / len;
  out[1] = y / len;
  out[2] = z / len;
}

uint32_t orc_encode_oct(const double v[3], int bits) { /* encoding.ts:33-47 */
  double l1 = fabs(v[0]) + fabs(v[1]) + fabs(v[2]);
  if (!(l1 > 0)) return 0;
  uint32_t max = (1u << bits) - 1u;
  uint32_t all_ones = max | (max << bits);
  double px = v[0] / l1, py = v[1] / l1;
  if (v[2] < 0) {
    double ax = fabs(px);
    px = (1.0 - fabs(py)) * (px >= 0 ? 1.0 : -1.0);
    py = (1.0 - ax) * (py >= 0 ? 1.0 : -1.0);
  }
  uint32_t code = (uint32_t)js_round((px * 0.5 + 0.5) * max) | ((uint32_t)js_round((py * 0.5 + 0.5) * max) << bits);
  return code == 0 ? all_ones : code;
}

/* A quaternion code: an octahedral axis of axis_bits + axis_bits, then the
   angle 0..pi in angle_bits (encoding.ts:73-111; QuatOct32 = 10 + 10 + 12,
   QuatOct24 = 8 + 8 + 8) */
void orc_decode_quat_oct(uint32_t code, int axis_bits, int angle_bits, double q[4]) {
  const uint32_t axis_mask = (uint32_t)((1ull << (2 * axis_bits)) - 1u);
  const uint32_t angle_max = (1u << angle_bits) - 1u;
  double axis[3];
  orc_decode_oct(code & axis_mask, axis_bits, axis);
  double angle = (double)((code >> (2 * axis_bits)) & angle_max) / (double)angle_max * PI;
  double s = sin(angle / 2.0);
  q[0] = axis[0] * s;
  q[1] = axis[1] * s;
  q[2] = axis[2] * s;
  q[3] = cos(angle / 2.0);
}

uint32_t orc_encode_quat_oct(const double q[4], int axis_bits, int angle_bits) {
  double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(len > 0)) return 0;
  double s = (q[3] < 0 ? -1.0 : 1.0) / len;
  double axis[3] = {q[0] * s, q[1] * s, q[2] * s};
  double angle = 2.0 * acos(fmin(1.0, q[3] * s));
  uint32_t angle_code = (uint32_t)js_round(angle / PI * (double)((1u << angle_bits) - 1u));
  return orc_encode_oct(axis, axis_bits) | (angle_code << (2 * axis_bits));
}

void orc_decode_quat_oct32(uint32_t code, double q[4]) { orc_decode_quat_oct(code, 10, 12, q); }

uint32_t orc_encode_quat_oct32(const double q[4]) { return orc_encode_quat_oct(q, 10, 12); }

static uint32_t encode_unorm8(double v) { /* encoding.ts:204-206 */
  double r = js_round(v * 255.0);
  return (uint32_t)(r < 0 ? 0 : (r > 255 ? 255 : r));
}

/* ---- spherical harmonics: src/core/sh.ts:362-407 ---- */

static const int SH_COEFFS[5] = {0, 3, 8, 15, 24}; /* sh.ts:59 */

void orc_sh_basis(const double d[3], double out[24]) {
  const double x = d[0], y = d[1], z = d[2];
  const double xx = x * x, yy = y * y, zz = z * z;
  out[0] = -0.4886025 * y;
  out[1] = 0.4886025 * z;
  out[2] = -0.4886025 * x;
  out[3] = 1.0925484 * x * y;
  out[4] = -1.0925484 * y * z;
  out[5] = 0.3153916 * (2 * zz - xx - yy);
  out[6] = -1.0925484 * x * z;
  out[7] = 0.5462742 * (xx - yy);
  out[8] = -0.5900436 * y * (3 * xx - yy);
  out[9] = 2.8906114 * x * y * z;
  out[10] = -0.4570458 * y * (4 * zz - xx - yy);
  out[11] = 0.3731763 * z * (2 * zz - 3 * xx - 3 * yy);
  out[12] = -0.4570458 * x * (4 * zz - xx - yy);
  out[13] = 1.4453057 * z * (xx - yy);
  out[14] = -0.5900436 * x * (xx - 3 * yy);
  out[15] = 2.5033429 * x * y * (xx - yy);
  out[16] = -1.7701308 * y * z * (3 * xx - yy);
  out[17] = 0.9461747 * x * y * (7 * zz - 1);
  out[18] = -0.6690465 * y * z * (7 * zz - 3);
  out[19] = 0.1057855 * (zz * (35 * zz - 30) + 3);
  out[20] = -0.6690465 * x * z * (7 * zz - 3);
  out[21] = 0.4730873 * (xx - yy) * (7 * zz - 1);
  out[22] = -1.7701308 * x * z * (xx - 3 * yy);
  out[23] = 0.6258357 * (xx * (xx - 3 * yy) - yy * (3 * xx - yy));
}

void orc_sh_evaluate(const double* c, const double dir[3], int degree, double out[3]) {
  double basis[24];
  orc_sh_basis(dir, basis);
  int deg = degree < 0 ? 0 : (degree > 4 ? 4 : degree);
  out[0] = out[1] = out[2] = 0.0;
  for (int k = 0; k < SH_COEFFS[deg]; k++) {
    out[0] += c[k * 3] * basis[k];
    out[1] += c[k * 3 + 1] * basis[k];
    out[2] += c[k * 3 + 2] * basis[k];
  }
}

/* ---- table rows ---- */

static double load_color(const rdx_table* t, uint64_t i, int j) {
  const int coeffs = 1 + SH_COEFFS[t->sh_degree];
  uint64_t at = i * (uint64_t)coeffs * 3 + (uint64_t)j;
  if (t->color_dtype == RDX_DTYPE_F16) {
    return orc_decode_half(((const uint16_t*)t->colors)[at]);
  }
  return (double)((const float*)t->colors)[at];
}

/* SH scale byte: 0 = zero, else 2^((code - 192) / 16) (sh.ts:70-87) */
static double decode_sh_scale(uint32_t code) { return code == 0 ? 0.0 : pow(2.0, ((double)code - 192.0) / 16.0); }

static uint32_t encode_sh_scale(double max) {
  if (!(max > 0)) return 0;
  double c = ceil(log2(max) * 16.0) + 192.0;
  uint32_t code = (uint32_t)(c < 1 ? 1 : (c > 255 ? 255 : c));
  while (code < 255 && decode_sh_scale(code) < max) code++;
  return code;
}

static const int PACKED_BAND_BYTES[4] = {10, 16, 22, 28}; /* sh.ts:62 */

/* Word j of splat i's SH entry: per-splat texel channels, or its palette
   entry (sh.tsl.ts:219-233; a label past the palette reads its last entry) */
static uint32_t sh_word(const rdx_table* t, uint64_t i, int j) {
  if (t->sh_palette) {
    uint64_t label = t->sh_label[i];
    if (t->sh_palette_size > 0 && label >= t->sh_palette_size) label = t->sh_palette_size - 1;
    return t->sh_palette[(label * t->sh_stride) * 4 + (uint64_t)j];
  }
  return t->ext_sh[j >> 2][i * 4 + (uint64_t)(j & 3)];
}

/* The coefficients of splat i's entry in the table's codec (sh.ts:137-170) */
static void load_sh_words(const rdx_table* t, uint64_t i, double* sh) {
  const int deg = t->sh_degree;
  if (t->sh_codec == RDX_SH_PACKED) {
    int byte = 0;
    for (int band = 0; band < deg; band++) {
      const int first = SH_COEFFS[band] * 3, end = SH_COEFFS[band + 1] * 3;
      uint32_t code = (sh_word(t, i, byte >> 2) >> ((byte & 3) * 8)) & 0xffu;
      double scale = decode_sh_scale(code) / 127.0;
      for (int v = first; v < end; v++) {
        int b = byte + 1 + v - first;
        int32_t sb = (int32_t)((sh_word(t, i, b >> 2) >> ((b & 3) * 8)) & 0xffu);
        if (sb > 127) sb -= 256;
        sh[v] = (double)sb * scale;
      }
      byte += PACKED_BAND_BYTES[band];
    }
  } else {
    for (int c = 0; c < SH_COEFFS[deg]; c++) orc_decode_ext_rgb(sh_word(t, i, c), &sh[c * 3]);
  }
}

static double decode_correlation(double e) { /* splats.ts:231-233 */
  return e == 0.0 ? 0.0 : (e > 0 ? -1.0 : 1.0) * exp(-fabs(e));
}

void orc_load_splat(const rdx_table* t, uint64_t i, orc_splat* s) {
  s->sh_degree = t->sh_degree;
  s->has_cov = 0;
  const int k = SH_COEFFS[t->sh_degree];
  if (t->layout == RDX_LAYOUT_EXT || t->layout == RDX_LAYOUT_COV) { /* splats.ts:188-197, 249-266 */
    const uint32_t* a = t->ext_a + i * 4;
    const uint32_t* b = t->ext_b + i * 4;
    for (int c = 0; c < 3; c++) {
      float f;
      memcpy(&f, &a[c], 4);
      s->center[c] = f;
    }
    s->opacity = (double)(a[3] >> 24) / 128.0; /* encoding.ts:213-215 */
    orc_decode_ext_rgb(b[0], s->rgb);
    if (t->layout == RDX_LAYOUT_EXT) {
      s->scales[0] = exp(orc_decode_half(b[1] & 0xffffu));
      s->scales[1] = exp(orc_decode_half(b[1] >> 16));
      s->scales[2] = exp(orc_decode_half(b[2] & 0xffffu));
      orc_decode_quat_oct32(b[3], s->quat);
    } else {
      const double xx = exp(orc_decode_half(b[1] & 0xffffu)), yy = exp(orc_decode_half(b[1] >> 16)),
                   zz = exp(orc_decode_half(b[2] & 0xffffu));
      s->cov[0] = xx;
      s->cov[1] = yy;
      s->cov[2] = zz;
      s->cov[3] = decode_correlation(orc_decode_half(b[2] >> 16)) * sqrt(xx * yy);
      s->cov[4] = decode_correlation(orc_decode_half(b[3] & 0xffffu)) * sqrt(xx * zz);
      s->cov[5] = decode_correlation(orc_decode_half(b[3] >> 16)) * sqrt(yy * zz);
      s->has_cov = 1;
      s->scales[0] = s->scales[1] = s->scales[2] = 1.0;
      s->quat[0] = s->quat[1] = s->quat[2] = 0.0;
      s->quat[3] = 1.0;
    }
    if (k) load_sh_words(t, i, s->sh);
  } else if (t->layout == RDX_LAYOUT_PACKED) { /* packedCodec.decode, splats.ts:288-306 */
    const uint32_t* p = t->packed + i * 4;
    const double rmin = t->packed_encoding[0], rmax = t->packed_encoding[1];
    const double lmin = t->packed_encoding[2], lmax = t->packed_encoding[3];
    const double range = rmax - rmin, step = (lmax - lmin) / 254.0;
    for (int c = 0; c < 3; c++) s->rgb[c] = rmin + ((double)((p[0] >> (8 * c)) & 0xffu) / 255.0) * range;
    s->opacity = (double)(p[0] >> 24) / 255.0;
    s->center[0] = orc_decode_half(p[1] & 0xffffu);
    s->center[1] = orc_decode_half(p[1] >> 16);
    s->center[2] = orc_decode_half(p[2] & 0xffffu);
    for (int c = 0; c < 3; c++) {
      uint32_t code = (p[3] >> (8 * c)) & 0xffu;
      s->scales[c] = code == 0 ? 0.0 : exp(lmin + (double)(code - 1) * step);
    }
    orc_decode_quat_oct((p[2] >> 16) | ((p[3] >> 24) << 16), 8, 8, s->quat);
    if (k) load_sh_words(t, i, s->sh);
  } else {
    for (int c = 0; c < 3; c++) {
      s->center[c] = t->centers[i * 3 + c];
      s->scales[c] = exp((double)t->log_scales[i * 3 + c]);
      s->rgb[c] = load_color(t, i, c);
    }
    for (int c = 0; c < 4; c++) s->quat[c] = t->quats[i * 4 + c];
    s->opacity = t->opacities[i];
    for (int c = 0; c < k * 3; c++) s->sh[c] = load_color(t, i, 3 + c);
  }
}

/* ---- 4x4 matrices, column-major ---- */

/* three.js multiplyMatrices: out = a * b, each sum left to right */
void orc_mat4_mul(const double a[16], const double b[16], double out[16]) {
  double r[16];
  for (int row = 0; row < 4; row++) {
    for (int col = 0; col < 4; col++) {
      double s = a[0 * 4 + row] * b[col * 4 + 0];
      s = s + a[1 * 4 + row] * b[col * 4 + 1];
      s = s + a[2 * 4 + row] * b[col * 4 + 2];
      s = s + a[3 * 4 + row] * b[col * 4 + 3];
      r[col * 4 + row] = s;
    }
  }
  memcpy(out, r, sizeof(r));
}

/* Inverse by the Laplace expansion in complementary 2x2 minors; 0 if singular */
int orc_mat4_invert(const double m[16], double out[16]) {
#define A(r, c) m[(c) * 4 + (r)]
  double s0 = A(0, 0) * A(1, 1) - A(1, 0) * A(0, 1);
  double s1 = A(0, 0) * A(1, 2) - A(1, 0) * A(0, 2);
  double s2 = A(0, 0) * A(1, 3) - A(1, 0) * A(0, 3);
  double s3 = A(0, 1) * A(1, 2) - A(1, 1) * A(0, 2);
  double s4 = A(0, 1) * A(1, 3) - A(1, 1) * A(0, 3);
  double s5 = A(0, 2) * A(1, 3) - A(1, 2) * A(0, 3);
  double c5 = A(2, 2) * A(3, 3) - A(3, 2) * A(2, 3);
  double c4 = A(2, 1) * A(3, 3) - A(3, 1) * A(2, 3);
  double c3 = A(2, 1) * A(3, 2) - A(3, 1) * A(2, 2);
  double c2 = A(2, 0) * A(3, 3) - A(3, 0) * A(2, 3);
  double c1 = A(2, 0) * A(3, 2) - A(3, 0) * A(2, 2);
  double c0 = A(2, 0) * A(3, 1) - A(3, 0) * A(2, 1);
  double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  if (det == 0.0) {
    memset(out, 0, 16 * sizeof(double));
    return 0;
  }
  double inv = 1.0 / det;
  double r[16];
#define R(rr, cc) r[(cc) * 4 + (rr)]
  R(0, 0) = (A(1, 1) * c5 - A(1, 2) * c4 + A(1, 3) * c3) * inv;
  R(0, 1) = (-A(0, 1) * c5 + A(0, 2) * c4 - A(0, 3) * c3) * inv;
  R(0, 2) = (A(3, 1) * s5 - A(3, 2) * s4 + A(3, 3) * s3) * inv;
  R(0, 3) = (-A(2, 1) * s5 + A(2, 2) * s4 - A(2, 3) * s3) * inv;
  R(1, 0) = (-A(1, 0) * c5 + A(1, 2) * c2 - A(1, 3) * c1) * inv;
  R(1, 1) = (A(0, 0) * c5 - A(0, 2) * c2 + A(0, 3) * c1) * inv;
  R(1, 2) = (-A(3, 0) * s5 + A(3, 2) * s2 - A(3, 3) * s1) * inv;
  R(1, 3) = (A(2, 0) * s5 - A(2, 2) * s2 + A(2, 3) * s1) * inv;
  R(2, 0) = (A(1, 0) * c4 - A(1, 1) * c2 + A(1, 3) * c0) * inv;
  R(2, 1) = (-A(0, 0) * c4 + A(0, 1) * c2 - A(0, 3) * c0) * inv;
  R(2, 2) = (A(3, 0) * s4 - A(3, 1) * s2 + A(3, 3) * s0) * inv;
  R(2, 3) = (-A(2, 0) * s4 + A(2, 1) * s2 - A(2, 3) * s0) * inv;
  R(3, 0) = (-A(1, 0) * c3 + A(1, 1) * c1 - A(1, 2) * c0) * inv;
  R(3, 1) = (A(0, 0) * c3 - A(0, 1) * c1 + A(0, 2) * c0) * inv;
  R(3, 2) = (-A(3, 0) * s3 + A(3, 1) * s1 - A(3, 2) * s0) * inv;
  R(3, 3) = (A(2, 0) * s3 - A(2, 1) * s1 + A(2, 2) * s0) * inv;
#undef R
#undef A
  memcpy(out, r, sizeof(r));
  return 1;
}

/* point transform without the w divide (the GPU's matrix.mul(vec4(c, 1)).xyz) */
static void xform_point(const double m[16], const double p[3], double out[3]) {
  double r[3];
  for (int row = 0; row < 3; row++) {
    double s = m[0 * 4 + row] * p[0];
    s = s + m[1 * 4 + row] * p[1];
    s = s + m[2 * 4 + row] * p[2];
    s = s + m[3 * 4 + row];
    r[row] = s;
  }
  out[0] = r[0];
  out[1] = r[1];
  out[2] = r[2];
}

static void clip_of(const double p[16], const double c[3], double clip[4]) {
  for (int row = 0; row < 4; row++) {
    double s = p[0 * 4 + row] * c[0];
    s = s + p[1 * 4 + row] * c[1];
    s = s + p[2 * 4 + row] * c[2];
    s = s + p[3 * 4 + row];
    clip[row] = s;
  }
}

/* 3x3 (row-major m[r][c]) helpers */
static void m3_mul(const double a[9], const double b[9], double out[9]) {
  double r[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] + a[i * 3 + 2] * b[2 * 3 + j];
  memcpy(out, r, sizeof(r));
}

static void m3_transpose(const double a[9], double out[9]) {
  double r[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r[i * 3 + j] = a[j * 3 + i];
  memcpy(out, r, sizeof(r));
}

/* mat3FromMat4 as row-major 3x3 */
static void m3_from_m4(const double m[16], double out[9]) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) out[r * 3 + c] = m[c * 4 + r];
}

void orc_params_default(rdx_params* p) { /* splatParams.ts:68-72 */
  p->max_std_dev = (float)sqrt(8.0);
  p->min_alpha = (float)(0.5 / 255.0);
  p->falloff = 1.0f;
  p->lod_inflate = 1;
  p->blur_amount = 0.3f;
  p->pre_blur_amount = 0.0f;
  p->clip_xy = 1.4f;
  p->min_pixel_radius = 0.0f;
  p->max_pixel_radius = 512.0f;
  p->min_contribution = 0.0f;
  p->focal_distance = 0.0f;
  p->aperture_tan = 0.0f;
  p->sort_guard = 0.0f;
  p->max_sh_degree = 4;
}

/* ---- word codecs: src/render/projection.tsl.ts:277-311 ---- */

static double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

static uint32_t encode_fixed16(double v) {
  return (uint32_t)clampd(floor((v + 2.0) / 4.0 * 65535.0 + 0.5), 0.0, 65535.0);
}

uint32_t orc_encode_depth20(double view_z) {
  float f32 = (float)(-view_z);
  uint32_t f;
  memcpy(&f, &f32, 4);
  const uint32_t lo = 113u << 23, hi = (145u << 23) - 1u;
  /* WGSL clamp on uint: f as unsigned (a negative depth has the sign bit set and clamps high) */
  f = f < lo ? lo : (f > hi ? hi : f);
  uint32_t code = (f - lo + 128u) >> 8;
  return code < 0xfffffu ? code : 0xfffffu;
}

uint32_t orc_encode_angle12(double angle) {
  return (uint32_t)floor(angle / PI * 4096.0 + 0.5) & 0xfffu;
}

static uint32_t encode_log_scale12(double scale) {
  const double top = 4094.0;
  double normalized = (clampd(log2(fmax(scale, 1e-20)), -4.0, 12.0) + 4.0) / 16.0 * top;
  return (uint32_t)clampd(floor(normalized + 0.5), 0.0, top) + 1u;
}

static uint32_t encode_opacity8(double opacity) {
  uint32_t v = (uint32_t)floor(clampd(opacity * 128.0, 0.0, 255.0) + 0.5);
  return v > 1u ? v : 1u;
}

/* ---- the projection ---- */

typedef struct eye_setup {
  double from_head[16];
  int identity;
  double proj[16];
  double from_head3[9];
  double focal[2];
  int ortho;
} eye_setup;

typedef struct object_setup {
  double a[16];        /* object -> head */
  double a3[9];
  double origin[3];    /* the head in object space (the view origin of the SH) */
  rdx_params params;
  uint64_t offset;
} object_setup;

static int mat_equal(const double a[16], const double b[16]) {
  for (int i = 0; i < 16; i++)
    if (a[i] != b[i]) return 0;
  return 1;
}

/* SH in object space from the view origin: splatGenerator.ts:152-158, sh.tsl.ts:255-266.
   A table with SH gets rgb + SH clamped at 0 even when the cap draws no band
   (GpuShReader.apply); a table without SH has no reader and no clamp. A splat
   at the view origin has no direction and gets no SH. */
static void splat_rgb(const orc_splat* s, const object_setup* o, double rgb[3]) {
  const rdx_params* p = &o->params;
  rgb[0] = s->rgb[0];
  rgb[1] = s->rgb[1];
  rgb[2] = s->rgb[2];
  int degree = s->sh_degree < p->max_sh_degree ? s->sh_degree : p->max_sh_degree;
  if (s->sh_degree >= 1) {
    double sh[3] = {0.0, 0.0, 0.0};
    if (degree >= 1) {
      double dv[3] = {s->center[0] - o->origin[0], s->center[1] - o->origin[1], s->center[2] - o->origin[2]};
      double len = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
      double dir[3] = {0, 0, 0};
      if (len > 0) {
        dir[0] = dv[0] / len;
        dir[1] = dv[1] / len;
        dir[2] = dv[2] / len;
      }
      orc_sh_evaluate(s->sh, dir, degree, sh);
    }
    for (int c = 0; c < 3; c++) rgb[c] = fmax(rgb[c] + sh[c], 0.0);
  }
}

/* One splat: outputs at index `gi` of the collection (n splats, E eyes) */
static void project_one(const orc_splat* s, const object_setup* o, const eye_setup* eyes, int n_eyes,
                        const rdx_camera* cam, int sort_bits, int cull_keys, uint64_t gi, uint64_t n,
                        const orc_outputs* out) {
  const rdx_params* p = &o->params;
  double rgb[3];
  splat_rgb(s, o, rgb);
  /* toCov: splats.tsl.ts:176-187, math.ts:12-45 */
  double qx = s->quat[0], qy = s->quat[1], qz = s->quat[2], qw = s->quat[3];
  double ql = sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
  if (!(ql > 0)) {
    qx = qy = qz = 0.0;
    qw = 1.0;
  } else {
    qx /= ql;
    qy /= ql;
    qz /= ql;
    qw /= ql;
  }
  const double sx = s->scales[0], sy = s->scales[1], sz = s->scales[2];
  /* M = R(q) diag(s) as row-major m[r][c]: column c is axis c scaled (math.tsl.ts:26-44) */
  double M[9] = {
      sx * (1 - 2 * (qy * qy + qz * qz)), sy * 2 * (qx * qy - qw * qz), sz * 2 * (qx * qz + qw * qy),
      sx * 2 * (qx * qy + qw * qz), sy * (1 - 2 * (qx * qx + qz * qz)), sz * 2 * (qy * qz - qw * qx),
      sx * 2 * (qx * qz - qw * qy), sy * 2 * (qy * qz + qw * qx), sz * (1 - 2 * (qx * qx + qy * qy)),
  };
  double Mt[9], cov[9];
  m3_transpose(M, Mt);
  m3_mul(M, Mt, cov);
  if (s->has_cov) { /* cov layout: the stored covariance (splats.tsl.ts:104-118) */
    const double c6[9] = {s->cov[0], s->cov[3], s->cov[4], s->cov[3], s->cov[1], s->cov[5], s->cov[4], s->cov[5], s->cov[2]};
    memcpy(cov, c6, sizeof(cov));
  }
  /* transformCov: splatTransform.tsl.ts:120-140 */
  double ch[3];
  xform_point(o->a, s->center, ch);
  double a3t[9], tmp[9], covh[9];
  m3_transpose(o->a3, a3t);
  m3_mul(o->a3, cov, tmp);
  m3_mul(tmp, a3t, covh);
  /* prepareSplat: projection.tsl.ts:42-64 */
  double opacity = s->opacity;
  double inflate = 1.0;
  if (opacity > 1.0) {
    opacity = fmin(opacity * 4.0 - 3.0, 5.0);
    if (p->lod_inflate) {
      inflate = pow(exp((opacity * opacity - 1.0) / E_CONST), 1.0 / 3.0);
      opacity = 1.0;
    }
  }
  for (int k = 0; k < 9; k++) covh[k] *= inflate * inflate;
  const double std_dev = opacity > 1.0 ? (double)p->max_std_dev + (opacity - 1.0) * 0.7 : (double)p->max_std_dev;
  /* cullInvisible: projection.tsl.ts:66-69 */
  const int degenerate = covh[0] == 0.0 && covh[4] == 0.0 && covh[8] == 0.0;
  const int invisible = opacity <= 0.0 || opacity < (double)p->min_alpha || degenerate;
  /* the head view (SplatProjection.ts:131-137): distance and sort guard */
  const double distance = sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
  int guarded = 1;
  if (p->sort_guard > 0.0f) { /* inSortGuard, projection.tsl.ts:145-155 (cov form) */
    double clip[4];
    clip_of(eyes[0].proj, ch, clip);
    double extent = sqrt(fmax(fmax(covh[0], covh[4]), covh[8]));
    double radius = extent * p->max_std_dev;
    double w = fmax(clip[3], 1e-6);
    double rx = eyes[0].proj[0] * radius / w, ry = eyes[0].proj[5] * radius / w;
    int inside = fabs(clip[0] / w) - rx <= (double)p->sort_guard + 1.0 && fabs(clip[1] / w) - ry <= (double)p->sort_guard + 1.0;
    int near_ = -ch[2] <= radius;
    guarded = ch[2] < radius && (inside || near_);
  }
  int any_visible = 0;
  for (int v = 0; v < n_eyes; v++) {
    const eye_setup* e = &eyes[v];
    /* splatInView: projection.tsl.ts:112-129 */
    double ce[3];
    if (e->identity) {
      ce[0] = ch[0];
      ce[1] = ch[1];
      ce[2] = ch[2];
    } else {
      xform_point(e->from_head, ch, ce);
    }
    double clip[4];
    clip_of(e->proj, ce, clip);
    double blur = p->blur_amount;
    if (p->focal_distance > 0.0f && p->aperture_tan > 0.0f && ce[2] < 0.0) {
      double depth = -ce[2];
      double coc_view = fabs(depth - (double)p->focal_distance) * (double)p->aperture_tan;
      double focal_pixels = cam->height * 0.5 * e->proj[5];
      double coc = e->ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
      blur = fmin(fmax(coc * coc, blur), (double)p->max_pixel_radius * p->max_pixel_radius);
    }
    double ndc[2] = {0.0, 0.0};
    if (clip[3] > 0.0) {
      ndc[0] = clip[0] / clip[3];
      ndc[1] = clip[1] / clip[3];
    }
    /* culls: projection.tsl.ts:132-140 */
    const double limit = fmin((double)p->clip_xy, 2.0) * clip[3];
    int ok = !(invisible || ce[2] >= 0.0 || clip[2] < cam->ndc_z_min * clip[3] || clip[2] >= clip[3] ||
               fabs(clip[0]) > limit || fabs(clip[1]) > limit);
    double a = 0, b = 0, d = 0, det = 0, opacity_c = 0, scale1 = 0, scale2 = 0, angle = 0;
    if (ok) {
      /* ewa.project: projections.tsl.ts:95-148 */
      double cov3[9];
      if (e->identity) {
        memcpy(cov3, covh, sizeof(cov3));
      } else {
        double ft[9], t2[9];
        m3_transpose(e->from_head3, ft);
        m3_mul(e->from_head3, covh, t2);
        m3_mul(t2, ft, cov3);
      }
      /* J as 3x3 (row-major), cov2D = J^T cov J with J's columns (J1x,0,J2x), (0,J1y,J2y), 0 */
      double J[9] = {0};
      if (e->ortho) {
        J[0] = e->focal[0];
        J[4] = e->focal[1];
      } else {
        double inv_z = 1.0 / ce[2];
        double j1x = e->focal[0] * inv_z, j1y = e->focal[1] * inv_z;
        double j2x = -(j1x * ce[0]) * inv_z, j2y = -(j1y * ce[1]) * inv_z;
        J[0 * 3 + 0] = j1x;
        J[1 * 3 + 1] = j1y;
        J[2 * 3 + 0] = j2x;
        J[2 * 3 + 1] = j2y;
      }
      double Jt[9], t3[9], cov2[9];
      m3_transpose(J, Jt);
      m3_mul(Jt, cov3, t3);
      m3_mul(t3, J, cov2);
      a = cov2[0] + p->pre_blur_amount;
      d = cov2[4] + p->pre_blur_amount;
      b = cov2[1];
      double det_orig = a * d - b * b;
      a += blur;
      d += blur;
      det = a * d - b * b;
      opacity_c = opacity * sqrt(fmax(0.0, det_orig / det));
      double contribution = opacity_c * 2.0 * PI * sqrt(fmax(0.0, det));
      /* boundFromCov: projection.tsl.ts:223-240 */
      double half = (a - d) * 0.5;
      double eigen1 = (a + d) * 0.5 + sqrt(half * half + b * b);
      double eigen2 = eigen1 > 0.0 ? fmax(det / eigen1, 0.0) : 0.0;
      scale1 = fmin((double)p->max_pixel_radius, std_dev * sqrt(fmax(eigen1, 0.0)));
      scale2 = fmin((double)p->max_pixel_radius, std_dev * sqrt(eigen2));
      int bound_ok = scale1 >= (double)p->min_pixel_radius || scale2 >= (double)p->min_pixel_radius;
      if (bound_ok) { /* eigenvector2: projection.tsl.ts:215-219 */
        double vx, vy;
        if (fabs(a - eigen1) >= fabs(d - eigen1)) {
          vx = b;
          vy = eigen1 - a;
        } else {
          vx = eigen1 - d;
          vy = b;
        }
        double len = sqrt(vx * vx + vy * vy);
        if (len > 0) {
          vx /= len;
          vy /= len;
        } else {
          vx = 1.0;
          vy = 0.0;
        }
        angle = atan2(vy, vx);
        if (angle < 0.0) angle += PI;
      }
      ok = opacity_c >= (double)p->min_alpha && contribution >= (double)p->min_contribution && bound_ok;
    }
    const uint64_t ei = (uint64_t)v * n + gi;
    if (out->visible) out->visible[ei] = (uint8_t)ok;
    if (ok) {
      if (out->mean2d) {
        out->mean2d[ei * 2 + 0] = (ndc[0] + 1.0) * 0.5 * cam->width;
        out->mean2d[ei * 2 + 1] = (ndc[1] + 1.0) * 0.5 * cam->height;
      }
      if (out->conic) {
        out->conic[ei * 3 + 0] = d / det;
        out->conic[ei * 3 + 1] = -b / det;
        out->conic[ei * 3 + 2] = a / det;
      }
      if (out->depth) out->depth[ei] = -ce[2];
      if (out->opacity) out->opacity[ei] = opacity_c;
      if (out->rgb)
        for (int c = 0; c < 3; c++) out->rgb[ei * 3 + c] = rgb[c];
      if (out->radii) {
        out->radii[ei * 3 + 0] = scale1;
        out->radii[ei * 3 + 1] = scale2;
        out->radii[ei * 3 + 2] = angle;
      }
      if (out->words) { /* projections.tsl.ts:135-140 */
        uint32_t* w = out->words + gi * (uint64_t)(4 * n_eyes) + (uint64_t)v * 4;
        double stored = opacity_c > 1.0 ? (opacity_c + 3.0) * 0.25 : opacity_c;
        w[0] = encode_fixed16(ndc[0]) | (encode_fixed16(ndc[1]) << 16);
        w[1] = orc_encode_depth20(ce[2]) | (orc_encode_angle12(angle) << 20);
        w[2] = orc_encode_ext_rgb(rgb);
        w[3] = encode_opacity8(stored) | (encode_log_scale12(scale1) << 8) | (encode_log_scale12(scale2) << 20);
      }
      any_visible = 1;
    } else {
      if (out->mean2d) out->mean2d[ei * 2] = out->mean2d[ei * 2 + 1] = 0.0;
      if (out->conic) out->conic[ei * 3] = out->conic[ei * 3 + 1] = out->conic[ei * 3 + 2] = 0.0;
      if (out->depth) out->depth[ei] = 0.0;
      if (out->opacity) out->opacity[ei] = 0.0;
      if (out->rgb) out->rgb[ei * 3] = out->rgb[ei * 3 + 1] = out->rgb[ei * 3 + 2] = 0.0;
      if (out->radii) out->radii[ei * 3] = out->radii[ei * 3 + 1] = out->radii[ei * 3 + 2] = 0.0;
      if (out->words) {
        uint32_t* w = out->words + gi * (uint64_t)(4 * n_eyes) + (uint64_t)v * 4;
        w[0] = w[1] = w[2] = w[3] = 0u;
      }
    }
  }
  /* SplatProjection.write: SplatProjection.ts:150-151 */
  const int keyed = cull_keys ? any_visible : (!invisible && guarded);
  if (out->keys) out->keys[gi] = keyed ? orc_sort_key(distance, sort_bits) : orc_invalid_key(sort_bits);
  if (out->distance) out->distance[gi] = distance;
}

/* SplatCamera.setViews (splatCamera.ts:119-138) and setTransforms
   (splatTransform.tsl.ts:78-107, splatGenerator.ts:105-112); returns the
   objects' set-ups (caller frees) and their total count */
static object_setup* setup_frame(const rdx_object* objects, int n_objects, const rdx_camera* cam,
                                 const rdx_params* params, eye_setup eyes[2], uint64_t* total) {
  double head_world[16];
  orc_mat4_invert(cam->head, head_world);
  for (int v = 0; v < cam->eyes; v++) {
    eye_setup* e = &eyes[v];
    e->identity = mat_equal(cam->eye[v].view, cam->head);
    if (e->identity) {
      memset(e->from_head, 0, sizeof(e->from_head));
      e->from_head[0] = e->from_head[5] = e->from_head[10] = e->from_head[15] = 1.0;
    } else {
      orc_mat4_mul(cam->eye[v].view, head_world, e->from_head);
    }
    m3_from_m4(e->from_head, e->from_head3);
    memcpy(e->proj, cam->eye[v].projection, sizeof(e->proj));
    e->focal[0] = cam->width * 0.5 * e->proj[0];
    e->focal[1] = cam->height * 0.5 * e->proj[5];
    e->ortho = cam->eye[v].ortho;
  }
  object_setup* objs = (object_setup*)calloc((size_t)(n_objects > 0 ? n_objects : 1), sizeof(object_setup));
  uint64_t n = 0;
  for (int i = 0; i < n_objects; i++) {
    object_setup* o = &objs[i];
    orc_mat4_mul(cam->head, objects[i].world, o->a);
    m3_from_m4(o->a, o->a3);
    double inv[16];
    orc_mat4_invert(o->a, inv);
    o->origin[0] = inv[12];
    o->origin[1] = inv[13];
    o->origin[2] = inv[14];
    o->params = objects[i].params ? *objects[i].params : *params;
    o->offset = n;
    n += objects[i].count;
  }
  *total = n;
  return objs;
}

int orc_project(const rdx_object* objects, int n_objects, const rdx_camera* cam, const rdx_params* params,
                int sort_bits, int cull_keys, int threads, const orc_outputs* out) {
  if (cam->eyes < 1 || cam->eyes > 2) return -1;
  eye_setup eyes[2];
  uint64_t n = 0;
  object_setup* objs = setup_frame(objects, n_objects, cam, params, eyes, &n);
#ifdef _OPENMP
  int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static, 4096) num_threads(nt)
#endif
  for (int64_t gi = 0; gi < (int64_t)n; gi++) {
    int oi = 0;
    while (oi + 1 < n_objects && (uint64_t)gi >= objs[oi + 1].offset) oi++;
    orc_splat s;
    orc_load_splat(objects[oi].table, (uint64_t)gi - objs[oi].offset, &s);
    project_one(&s, &objs[oi], eyes, cam->eyes, cam, sort_bits, cull_keys, (uint64_t)gi, n, out);
  }
  free(objs);
  return 0;
}

/* ---- the ray projection methods: src/render/projections.tsl.ts:170-474 ---- */

static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* quatRotate (src/gpu/math.tsl.ts:12-15): v + w t + q.xyz x t with t = 2 q.xyz x v */
static void quat_rotate(const double q[4], const double v[3], double out[3]) {
  const double t[3] = {2.0 * (q[1] * v[2] - q[2] * v[1]), 2.0 * (q[2] * v[0] - q[0] * v[2]),
                       2.0 * (q[0] * v[1] - q[1] * v[0])};
  const double r[3] = {v[0] + q[3] * t[0] + (q[1] * t[2] - q[2] * t[1]), v[1] + q[3] * t[1] + (q[2] * t[0] - q[0] * t[2]),
                       v[2] + q[3] * t[2] + (q[0] * t[1] - q[1] * t[0])};
  memcpy(out, r, sizeof(r));
}

/* quatMul (math.tsl.ts:17-23): a applied after b */
static void quat_mul(const double a[4], const double b[4], double out[4]) {
  const double r[4] = {a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
                       a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
                       a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3],
                       a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]};
  memcpy(out, r, sizeof(r));
}

static void quat_normalize(const double q[4], double out[4]) { /* a zero quaternion: the identity */
  const double l = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(l > 0)) {
    out[0] = out[1] = out[2] = 0.0;
    out[3] = 1.0;
    return;
  }
  for (int k = 0; k < 4; k++) out[k] = q[k] / l;
}

/* The unit quaternion of a rotation matrix (row-major), by the trace and the
   largest diagonal element (Shoemake's method), as three.js Matrix4.decompose
   finds the quaternions of setTransform (splatTransform.tsl.ts:64-74) and
   SplatCamera.setViews (splatCamera.ts:129-131) */
static void rotation_to_quat(const double m[9], double q[4]) {
  const double tr = m[0] + m[4] + m[8];
  if (tr > 0.0) {
    const double s = 0.5 / sqrt(tr + 1.0);
    q[3] = 0.25 / s;
    q[0] = (m[7] - m[5]) * s;
    q[1] = (m[2] - m[6]) * s;
    q[2] = (m[3] - m[1]) * s;
  } else if (m[0] > m[4] && m[0] > m[8]) {
    const double s = 2.0 * sqrt(1.0 + m[0] - m[4] - m[8]);
    q[3] = (m[7] - m[5]) / s;
    q[0] = 0.25 * s;
    q[1] = (m[1] + m[3]) / s;
    q[2] = (m[2] + m[6]) / s;
  } else if (m[4] > m[8]) {
    const double s = 2.0 * sqrt(1.0 + m[4] - m[0] - m[8]);
    q[3] = (m[2] - m[6]) / s;
    q[0] = (m[1] + m[3]) / s;
    q[1] = 0.25 * s;
    q[2] = (m[5] + m[7]) / s;
  } else {
    const double s = 2.0 * sqrt(1.0 + m[8] - m[0] - m[4]);
    q[3] = (m[3] - m[1]) / s;
    q[0] = (m[2] + m[6]) / s;
    q[1] = (m[5] + m[7]) / s;
    q[2] = 0.25 * s;
  }
}

static double det3_cols(const double* c0, const double* c1, const double* c2) {
  return c0[0] * (c1[1] * c2[2] - c1[2] * c2[1]) - c1[0] * (c0[1] * c2[2] - c0[2] * c2[1]) +
         c2[0] * (c0[1] * c1[2] - c0[2] * c1[1]);
}

/* The rotation of a column-major 4x4's 3x3 part (columns divided by their
   lengths, the first negated when the determinant is negative) as a quaternion */
static void decompose_quat(const double m[16], double q[4]) {
  const double* c[3] = {m, m + 4, m + 8};
  double len[3] = {sqrt(dot3(c[0], c[0])), sqrt(dot3(c[1], c[1])), sqrt(dot3(c[2], c[2]))};
  if (det3_cols(c[0], c[1], c[2]) < 0.0) len[0] = -len[0];
  double r[9];
  for (int row = 0; row < 3; row++)
    for (int col = 0; col < 3; col++) r[row * 3 + col] = c[col][row] / len[col];
  rotation_to_quat(r, q);
}

/* isUniformScale (splatTransform.tsl.ts:46-62) of the object -> head matrix:
   with G = M^T M and s2 = trace(G) / 3, every entry of G - s2 I within 1e-6 s2
   and det(M) > 0; then the rotation and |det(M)|^(1/3) (setTransform, 64-74) */
static int uniform_transform(const double a[16], double q[4], double* scale) {
  const double* c[3] = {a, a + 4, a + 8};
  const double s2 = (dot3(c[0], c[0]) + dot3(c[1], c[1]) + dot3(c[2], c[2])) / 3.0;
  if (!(s2 > 0)) return 0;
  for (int i = 0; i < 3; i++)
    for (int j = i; j < 3; j++)
      if (fabs(dot3(c[i], c[j]) - (i == j ? s2 : 0.0)) > 1e-6 * s2) return 0;
  const double det = det3_cols(c[0], c[1], c[2]);
  if (!(det > 0)) return 0;
  decompose_quat(a, q);
  *scale = cbrt(fabs(det));
  return 1;
}

/* basisToQuat (math.tsl.ts:117-150): the w >= 0 quaternion of the orthonormal
   columns x, y, z */
static void basis_to_quat(const double x[3], const double y[3], const double z[3], double q[4]) {
  double four, inv;
  if (z[2] <= 0.0) {
    const double dif10 = y[1] - x[0], omm22 = 1.0 - z[2];
    if (dif10 <= 0.0) {
      four = omm22 - dif10;
      inv = 0.5 / sqrt(fmax(four, 1e-30));
      q[0] = four * inv, q[1] = (x[1] + y[0]) * inv, q[2] = (x[2] + z[0]) * inv, q[3] = (y[2] - z[1]) * inv;
    } else {
      four = omm22 + dif10;
      inv = 0.5 / sqrt(fmax(four, 1e-30));
      q[0] = (x[1] + y[0]) * inv, q[1] = four * inv, q[2] = (y[2] + z[1]) * inv, q[3] = (z[0] - x[2]) * inv;
    }
  } else {
    const double sum10 = y[1] + x[0], opm22 = 1.0 + z[2];
    if (sum10 <= 0.0) {
      four = opm22 - sum10;
      inv = 0.5 / sqrt(fmax(four, 1e-30));
      q[0] = (x[2] + z[0]) * inv, q[1] = (y[2] + z[1]) * inv, q[2] = four * inv, q[3] = (x[1] - y[0]) * inv;
    } else {
      four = opm22 + sum10;
      inv = 0.5 / sqrt(fmax(four, 1e-30));
      q[0] = (y[2] - z[1]) * inv, q[1] = (z[0] - x[2]) * inv, q[2] = (x[1] - y[0]) * inv, q[3] = four * inv;
    }
  }
  const double l = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (int k = 0; k < 4; k++) q[k] /= l;
  if (q[3] < 0.0)
    for (int k = 0; k < 4; k++) q[k] = -q[k];
}

/* scaleQuatMatrix (math.tsl.ts:25-44): column k is axis k of R(q) times s[k] */
static void scale_quat_cols(const double s[3], const double q[4], double col[3][3]) {
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  col[0][0] = s[0] * (1.0 - 2.0 * (y * y + z * z));
  col[0][1] = s[0] * (2.0 * (x * y + w * z));
  col[0][2] = s[0] * (2.0 * (x * z - w * y));
  col[1][0] = s[1] * (2.0 * (x * y - w * z));
  col[1][1] = s[1] * (1.0 - 2.0 * (x * x + z * z));
  col[1][2] = s[1] * (2.0 * (y * z + w * x));
  col[2][0] = s[2] * (2.0 * (x * z + w * y));
  col[2][1] = s[2] * (2.0 * (y * z - w * x));
  col[2][2] = s[2] * (1.0 - 2.0 * (x * x + y * y));
}

/* symEigens (math.tsl.ts:46-112): Jacobi rotations on the symmetric matrix
   (xx, yy, zz | xy, xz, yz), at most 16, stopping once every off-diagonal
   element is within 1e-6 of the diagonal's absolute sum; eigenvalues
   descending, eigenvectors right-handed. A[c][r] and V[c][r] are column c,
   row r, as the reference indexes them. */
static void sym_eigens(const double d[3], const double o[3], double values[3], double vec[3][3]) {
  const double eps = 1e-6 * (fabs(d[0]) + fabs(d[1]) + fabs(d[2]));
  double A[3][3] = {{d[0], o[0], o[1]}, {o[0], d[1], o[2]}, {o[1], o[2], d[2]}};
  double V[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  for (int it = 0; it < 16; it++) {
    int p = 0, q = 1;
    double mx = fabs(A[0][1]);
    if (fabs(A[0][2]) > mx) {
      mx = fabs(A[0][2]);
      q = 2;
    }
    if (fabs(A[1][2]) > mx) {
      mx = fabs(A[1][2]);
      p = 1;
      q = 2;
    }
    if (mx <= eps) break;
    const double phi = atan2(A[p][q] * 2.0, A[q][q] - A[p][p]) * 0.5;
    const double c = cos(phi), sn = sin(phi);
    for (int r = 0; r < 3; r++) {
      const double x = A[r][p], y = A[r][q];
      A[r][p] = c * x - sn * y;
      A[r][q] = sn * x + c * y;
    }
    for (int r = 0; r < 3; r++) {
      const double x = A[p][r], y = A[q][r];
      A[p][r] = c * x - sn * y;
      A[q][r] = sn * x + c * y;
    }
    A[p][q] = 0.0;
    A[q][p] = 0.0;
    for (int r = 0; r < 3; r++) {
      const double x = V[r][p], y = V[r][q];
      V[r][p] = c * x - sn * y;
      V[r][q] = sn * x + c * y;
    }
  }
  double l[3] = {A[0][0], A[1][1], A[2][2]};
  double v[3][3];
  for (int i = 0; i < 3; i++) {
    const double w[3] = {V[0][i], V[1][i], V[2][i]};
    const double len = sqrt(dot3(w, w));
    for (int k = 0; k < 3; k++) v[i][k] = w[k] / len;
  }
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int k = 0; k < 3; k++) {
    const int i = pairs[k][0], j = pairs[k][1];
    if (l[i] < l[j]) {
      const double t = l[i];
      l[i] = l[j];
      l[j] = t;
      double w[3];
      memcpy(w, v[i], sizeof(w));
      memcpy(v[i], v[j], sizeof(w));
      memcpy(v[j], w, sizeof(w));
    }
  }
  const double cr[3] = {v[0][1] * v[1][2] - v[0][2] * v[1][1], v[0][2] * v[1][0] - v[0][0] * v[1][2],
                        v[0][0] * v[1][1] - v[0][1] * v[1][0]};
  if (dot3(cr, v[2]) < 0.0)
    for (int k = 0; k < 3; k++) v[2][k] = -v[2][k];
  memcpy(values, l, sizeof(l));
  memcpy(vec, v, sizeof(v));
}

/* The splat form of a head-space covariance (row-major): fromCov
   (src/gpu/splats.tsl.ts:189-199), scales sqrt(max(eigenvalue, 0)) and the
   rotation of the eigenvector basis */
static void from_cov(const double cov[9], double scales[3], double q[4]) {
  const double d[3] = {cov[0], cov[4], cov[8]}, o[3] = {cov[3], cov[6], cov[7]};
  double values[3], v[3][3];
  sym_eigens(d, o, values, v);
  for (int k = 0; k < 3; k++) scales[k] = sqrt(fmax(values[k], 0.0));
  basis_to_quat(v[0], v[1], v[2], q);
}

/* P (column-major) times (v, 0) */
static void proj_dir(const double p[16], const double v[3], double out[4]) {
  for (int row = 0; row < 4; row++) {
    double s = p[0 * 4 + row] * v[0];
    s = s + p[1 * 4 + row] * v[1];
    s = s + p[2 * 4 + row] * v[2];
    out[row] = s;
  }
}

typedef struct orc_bound { /* Bound, projection.tsl.ts:206-210 */
  double ndc[2], angle, scales[2];
} orc_bound;

/* eigenvector2 (projection.tsl.ts:215-219) */
static void eigenvector2(double a, double b, double d, double eig, double v[2]) {
  double vx, vy;
  if (fabs(a - eig) >= fabs(d - eig)) {
    vx = b;
    vy = eig - a;
  } else {
    vx = eig - d;
    vy = b;
  }
  const double len = sqrt(vx * vx + vy * vy);
  v[0] = len > 0.0 ? vx / len : 1.0;
  v[1] = len > 0.0 ? vy / len : 0.0;
}

/* boundFromCov (projection.tsl.ts:223-240) */
static int bound_from_cov(double a, double b, double d, double std_dev, const rdx_params* p, orc_bound* bd) {
  const double det = a * d - b * b;
  const double half = (a - d) * 0.5;
  const double eigen1 = (a + d) * 0.5 + sqrt(half * half + b * b);
  const double eigen2 = eigen1 > 0.0 ? fmax(det / eigen1, 0.0) : 0.0;
  const double scale1 = fmin((double)p->max_pixel_radius, std_dev * sqrt(fmax(eigen1, 0.0)));
  const double scale2 = fmin((double)p->max_pixel_radius, std_dev * sqrt(eigen2));
  const int ok = scale1 >= (double)p->min_pixel_radius || scale2 >= (double)p->min_pixel_radius;
  if (ok) {
    double v[2];
    eigenvector2(a, b, d, eigen1, v);
    const double angle = atan2(v[1], v[0]);
    bd->angle = angle < 0.0 ? angle + PI : angle;
    bd->scales[0] = scale1;
    bd->scales[1] = scale2;
  }
  return ok;
}

/* screenBound (projection.tsl.ts:243-247) */
static void screen_bound(const rdx_camera* cam, const rdx_params* p, orc_bound* bd) {
  bd->ndc[0] = bd->ndc[1] = 0.0;
  bd->angle = 0.0;
  bd->scales[0] = bd->scales[1] = fmin((double)p->max_pixel_radius, sqrt(cam->width * cam->width + cam->height * cam->height) * 0.5);
}

/* clipBoundToScreen (projection.tsl.ts:250-273) */
static int clip_bound_to_screen(const rdx_camera* cam, orc_bound* bd) {
  const double hx = cam->width * 0.5, hy = cam->height * 0.5;
  const double ca = cos(bd->angle), sa = sin(bd->angle);
  const double cx = ca * bd->scales[0], cy = ca * bd->scales[1], sx = sa * bd->scales[0], sy = sa * bd->scales[1];
  const double ex = sqrt(cx * cx + sy * sy), ey = sqrt(sx * sx + cy * cy);
  const double mx = bd->ndc[0] * hx, my = bd->ndc[1] * hy;
  double lox = mx - ex, loy = my - ey, hix = mx + ex, hiy = my + ey;
  if (!(lox >= -hx && loy >= -hy && hix <= hx && hiy <= hy)) {
    lox = fmax(lox, -hx);
    loy = fmax(loy, -hy);
    hix = fmin(hix, hx);
    hiy = fmin(hiy, hy);
    if (lox >= hix || loy >= hiy) return 0;
    bd->ndc[0] = (lox + hix) * 0.5 / hx;
    bd->ndc[1] = (loy + hiy) * 0.5 / hy;
    bd->angle = 0.0;
    bd->scales[0] = (hix - lox) * 0.5;
    bd->scales[1] = (hiy - loy) * 0.5;
  }
  return 1;
}

/* encodeLogScale (projection.tsl.ts:299-303) in `bits`, rounded up when outward */
static uint32_t encode_log_scale_bits(double scale, int bits, int outward) {
  const double top = (double)((1u << bits) - 2u);
  const double normalized = (clampd(log2(fmax(scale, 1e-20)), -4.0, 12.0) + 4.0) / 16.0 * top;
  return (uint32_t)clampd(outward ? ceil(normalized) : floor(normalized + 0.5), 0.0, top) + 1u;
}

/* encodeBound (projection.tsl.ts:352-360): NDC 2x16; 10-bit angle | 2 x 11-bit
   log2 scales rounded outward, widened by the angle's half step */
static void encode_bound(const orc_bound* bd, uint32_t w[2]) {
  const uint32_t angle_code = (uint32_t)floor(bd->angle / PI * 1024.0 + 0.5) & 1023u;
  const double slack = fmax(bd->scales[0], bd->scales[1]) * (sin(PI / 1024.0 / 2.0) * 1.001);
  w[0] = encode_fixed16(bd->ndc[0]) | (encode_fixed16(bd->ndc[1]) << 16);
  w[1] = angle_code | (encode_log_scale_bits(bd->scales[0] + slack, 11, 1) << 10) |
         (encode_log_scale_bits(bd->scales[1] + slack, 11, 1) << 21);
}

/* encodeCenter (projection.tsl.ts:317-332): [direction's top 16 + 16 bits,
   float32 distance, low 4 + 4 bits at bits 24-31] */
static void encode_center(const double c[3], uint32_t w[3]) {
  const double distance = sqrt(dot3(c, c));
  const double l1 = fmax(fabs(c[0]) + fabs(c[1]) + fabs(c[2]), 1e-30);
  double px = c[0] / l1, py = c[1] / l1;
  const double sx = px >= 0.0 ? 1.0 : -1.0, sy = py >= 0.0 ? 1.0 : -1.0;
  if (c[2] < 0.0) {
    const double ax = fabs(px);
    px = (1.0 - fabs(py)) * sx;
    py = (1.0 - ax) * sy;
  }
  const uint32_t qx = (uint32_t)floor((px * 0.5 + 0.5) * 1048575.0 + 0.5);
  const uint32_t qy = (uint32_t)floor((py * 0.5 + 0.5) * 1048575.0 + 0.5);
  const float df = (float)distance;
  uint32_t db;
  memcpy(&db, &df, 4);
  w[0] = (qx >> 4) | ((qy >> 4) << 16);
  w[1] = db;
  w[2] = ((qx & 15u) << 24) | (qy << 28);
}

/* gutBound (projections.tsl.ts:183-220): the unscented transform of 7 sigma points */
static int gut_bound(const double ce[3], const eye_setup* e, const double q[4], const double s[3], double std_dev,
                     const rdx_params* p, const rdx_camera* cam, orc_bound* bd) {
  const double r3 = sqrt(3.0);
  const double ss[3] = {s[0] * r3, s[1] * r3, s[2] * r3};
  double col[3][3];
  scale_quat_cols(ss, q, col);
  const double hx = cam->width * 0.5, hy = cam->height * 0.5;
  double px[7], py[7];
  int in_front = 1;
  for (int i = 0; i < 7; i++) {
    double pt[3] = {ce[0], ce[1], ce[2]};
    if (i > 0) {
      const double sign = (i & 1) ? 1.0 : -1.0;
      for (int k = 0; k < 3; k++) pt[k] = ce[k] + sign * col[(i - 1) / 2][k];
    }
    double clip[4];
    clip_of(e->proj, pt, clip);
    in_front = in_front && clip[3] > 0.0;
    px[i] = clip[0] / clip[3] * hx;
    py[i] = clip[1] / clip[3] * hy;
  }
  if (!in_front) {
    screen_bound(cam, p, bd);
    return 1;
  }
  const double sixth = 1.0 / 6.0;
  double mx = 0.0, my = 0.0;
  for (int i = 1; i < 7; i++) {
    mx += px[i] * sixth;
    my += py[i] * sixth;
  }
  const double d0x = px[0] - mx, d0y = py[0] - my;
  double a = d0x * d0x * 2.0, b = d0x * d0y * 2.0, d = d0y * d0y * 2.0;
  for (int i = 1; i < 7; i++) {
    const double dx = px[i] - mx, dy = py[i] - my;
    a += dx * dx * sixth;
    b += dx * dy * sixth;
    d += dy * dy * sixth;
  }
  const int ok = bound_from_cov(a, b, d, std_dev, p, bd);
  bd->ndc[0] = mx / hx;
  bd->ndc[1] = my / hy;
  return ok;
}

/* htgsBound (projections.tsl.ts:223-262): the exact outline of the std-dev ellipsoid */
static int htgs_bound(const double ce[3], const double ndc[2], const eye_setup* e, const double q[4], const double s[3],
                      double std_dev, const rdx_params* p, const rdx_camera* cam, orc_bound* bd) {
  const double ss[3] = {s[0] * std_dev, s[1] * std_dev, s[2] * std_dev};
  double col[3][3], T[3][4], c3[4];
  scale_quat_cols(ss, q, col);
  for (int k = 0; k < 3; k++) proj_dir(e->proj, col[k], T[k]);
  clip_of(e->proj, ce, c3);
  const double xs[3] = {T[0][0], T[1][0], T[2][0]}, ys[3] = {T[0][1], T[1][1], T[2][1]},
               ws[3] = {T[0][3], T[1][3], T[2][3]};
  const double qww = dot3(ws, ws) - c3[3] * c3[3];
  int valid = qww < 0.0 && c3[3] > 0.0;
  double cx = 0.0, cy = 0.0, a = 0.0, b = 0.0, d = 0.0;
  if (valid) {
    double u[3], v[3];
    for (int k = 0; k < 3; k++) {
      u[k] = xs[k] * c3[3] - ws[k] * c3[0];
      v[k] = ys[k] * c3[3] - ws[k] * c3[1];
    }
    const double sww = dot3(ws, ws), xw = dot3(xs, ws), yw = dot3(ys, ws);
    const double inv_c2 = 1.0 / (qww * qww);
    const double hx = cam->width * 0.5, hy = cam->height * 0.5;
    a = (dot3(u, u) - (sww * dot3(xs, xs) - xw * xw)) * inv_c2 * hx * hx;
    b = (dot3(u, v) - (sww * dot3(xs, ys) - xw * yw)) * inv_c2 * hx * hy;
    d = (dot3(v, v) - (sww * dot3(ys, ys) - yw * yw)) * inv_c2 * hy * hy;
    cx = ndc[0] + dot3(ws, u) / (c3[3] * qww);
    cy = ndc[1] + dot3(ws, v) / (c3[3] * qww);
    valid = a > 0.0 && d > 0.0 && a * d - b * b > 0.0;
  }
  if (!valid) {
    screen_bound(cam, p, bd);
    return 1;
  }
  const int ok = bound_from_cov(a, b, d, 1.0, p, bd);
  bd->ndc[0] = cx;
  bd->ndc[1] = cy;
  return ok;
}

/* quadOffScreen (projections.tsl.ts:336-352) */
static int quad_off_screen(const double proj[16], const double mu[3], const double a0[3], const double a1[3]) {
  double c[4], p0[4], p1[4];
  clip_of(proj, mu, c);
  proj_dir(proj, a0, p0);
  proj_dir(proj, a1, p1);
  int in_front = 1, o0 = 1, o1 = 1, o2 = 1, o3 = 1;
  for (int i = 0; i < 4; i++) {
    double clip[4];
    for (int k = 0; k < 4; k++) clip[k] = c[k] + ((i & 1) ? p0[k] : -p0[k]) + ((i & 2) ? p1[k] : -p1[k]);
    in_front = in_front && clip[3] > 0.0;
    o0 = o0 && clip[0] < -clip[3];
    o1 = o1 && clip[0] > clip[3];
    o2 = o2 && clip[1] < -clip[3];
    o3 = o3 && clip[1] > clip[3];
  }
  return in_front && (o0 || o1 || o2 || o3);
}

/* raygsFrame (projections.tsl.ts:356-397): the quad facing the eye */
static int raygs_frame(const double ce[3], const eye_setup* e, const double q[4], const double s[3], double std_dev,
                       double fq[4], double lengths[2], double* c2_out) {
  int ok = 1;
  const double kappa = std_dev * std_dev;
  const double conj[4] = {-q[0], -q[1], -q[2], q[3]};
  double local[3], mu[3];
  quat_rotate(conj, ce, local);
  for (int k = 0; k < 3; k++) local[k] /= s[k];
  double c2 = dot3(local, local);
  if (e->ortho) {
    const double back[3] = {0.0, 0.0, -1.0};
    double v[3];
    quat_rotate(conj, back, v);
    for (int k = 0; k < 3; k++) v[k] /= s[k];
    const double l = sqrt(dot3(v, v));
    for (int k = 0; k < 3; k++) mu[k] = v[k] / l;
    c2 = 1e18;
  } else {
    ok = c2 > kappa * 1.0001;
    const double inv = 1.0 / sqrt(c2);
    for (int k = 0; k < 3; k++) mu[k] = local[k] * inv;
  }
  const double t[3] = {mu[0], mu[1], mu[2] + (mu[2] >= 0.0 ? 1.0 : -1.0)};
  const double inv_den = 2.0 / dot3(t, t);
  const double v0[3] = {s[0] * (t[0] * (t[0] * inv_den) - 1.0), s[1] * (t[1] * (t[0] * inv_den)),
                        s[2] * (t[2] * (t[0] * inv_den))};
  const double v1[3] = {s[0] * (t[0] * (t[1] * inv_den)), s[1] * (t[1] * (t[1] * inv_den) - 1.0),
                        s[2] * (t[2] * (t[1] * inv_den))};
  double q0[3], q1[3];
  quat_rotate(q, v0, q0);
  quat_rotate(q, v1, q1);
  const double bxx = dot3(q0, q0), bxy = dot3(q0, q1), byy = dot3(q1, q1);
  const double diff = bxx - byy;
  const double eig1 = (bxx + byy) * 0.5 + sqrt(fmax(0.0, diff * diff * 0.25 + bxy * bxy));
  double u1[2];
  eigenvector2(bxx, bxy, byy, eig1, u1);
  const double u0[2] = {-u1[1], u1[0]};
  double axis0[3], axis1[3];
  for (int k = 0; k < 3; k++) {
    axis0[k] = q0[k] * u0[0] + q1[k] * u0[1];
    axis1[k] = q0[k] * u1[0] + q1[k] * u1[1];
  }
  lengths[0] = sqrt(dot3(axis0, axis0));
  lengths[1] = sqrt(dot3(axis1, axis1));
  ok = ok && lengths[0] > 0.0 && lengths[1] > 0.0;
  const double z_scale = std_dev / sqrt(fmax(1.0 - kappa / c2, 1e-4));
  double za0[3], za1[3];
  for (int k = 0; k < 3; k++) {
    za0[k] = axis0[k] * z_scale;
    za1[k] = axis1[k] * z_scale;
  }
  ok = ok && !quad_off_screen(e->proj, ce, za0, za1);
  double n0[3], n1[3], n2[3];
  for (int k = 0; k < 3; k++) {
    n0[k] = axis0[k] / lengths[0];
    n1[k] = axis1[k] / lengths[1];
  }
  n2[0] = n0[1] * n1[2] - n0[2] * n1[1];
  n2[1] = n0[2] * n1[0] - n0[0] * n1[2];
  n2[2] = n0[0] * n1[1] - n0[1] * n1[0];
  basis_to_quat(n0, n1, n2, fq);
  *c2_out = c2;
  return ok;
}

/* One splat of a ray method: its head and eye words (row `gi`) and its key
   (SplatProjection.project/write, SplatProjection.ts:126-153; rayProjection
   and raygs, projections.tsl.ts:266-333, 399-467) */
static void rays_one(const orc_splat* s, const object_setup* o, const eye_setup* eyes, const double eye_q[2][4],
                     int n_eyes, const rdx_camera* cam, int method, const double tq[4], double tscale, int uniform,
                     int sort_bits, int cull_keys, uint64_t gi, uint32_t* words, uint32_t* keys) {
  const rdx_params* p = &o->params;
  const int head_words = method == ORC_METHOD_RAYGS ? 4 : 6, eye_words = method == ORC_METHOD_RAYGS ? 3 : 2;
  uint32_t* row = words ? words + gi * (uint64_t)(head_words + n_eyes * eye_words) : NULL;
  double rgb[3];
  splat_rgb(s, o, rgb);
  double ch[3], qn[4], qh[4], sc[3];
  xform_point(o->a, s->center, ch);
  quat_normalize(s->quat, qn);
  if (uniform && !s->has_cov) { /* transformUniform (splatTransform.tsl.ts:143-152) */
    quat_mul(tq, qn, qh);
    for (int k = 0; k < 3; k++) sc[k] = s->scales[k] * tscale;
  } else {
    /* transformSplat's other branch (toCov, transformCov, fromCov: splatTransform.tsl.ts:117-162,
       splats.tsl.ts:176-199), or a cov table's transformCov and fromCov (transformForm, convertForm) */
    double cov[9];
    if (s->has_cov) {
      const double c6[9] = {s->cov[0], s->cov[3], s->cov[4], s->cov[3], s->cov[1], s->cov[5], s->cov[4], s->cov[5], s->cov[2]};
      memcpy(cov, c6, sizeof(cov));
    } else {
      double col[3][3], M[9], Mt[9];
      scale_quat_cols(s->scales, qn, col);
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) M[r * 3 + c] = col[c][r];
      m3_transpose(M, Mt);
      m3_mul(M, Mt, cov);
    }
    double a3t[9], tmp[9], covh[9];
    m3_transpose(o->a3, a3t);
    m3_mul(o->a3, cov, tmp);
    m3_mul(tmp, a3t, covh);
    from_cov(covh, sc, qh);
  }
  /* prepareSplat, splat form (projection.tsl.ts:42-64) */
  double opacity = s->opacity, inflate = 1.0;
  if (opacity > 1.0) {
    opacity = fmin(opacity * 4.0 - 3.0, 5.0);
    if (p->lod_inflate) {
      inflate = pow(exp((opacity * opacity - 1.0) / E_CONST), 1.0 / 3.0);
      opacity = 1.0;
    }
  }
  for (int k = 0; k < 3; k++) sc[k] *= inflate;
  const double std_dev = opacity > 1.0 ? (double)p->max_std_dev + (opacity - 1.0) * 0.7 : (double)p->max_std_dev;
  const int invisible = opacity <= 0.0 || opacity < (double)p->min_alpha || (sc[0] == 0.0 && sc[1] == 0.0 && sc[2] == 0.0);
  /* the head: splatInView(headFrame()), eye 0's lens */
  const eye_setup* e0 = &eyes[0];
  double hclip[4];
  clip_of(e0->proj, ch, hclip);
  double hblur = p->blur_amount;
  if (p->focal_distance > 0.0f && p->aperture_tan > 0.0f && ch[2] < 0.0) {
    const double depth = -ch[2];
    const double coc_view = fabs(depth - (double)p->focal_distance) * (double)p->aperture_tan;
    const double focal_pixels = cam->height * 0.5 * e0->proj[5];
    const double coc = e0->ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
    hblur = fmin(fmax(coc * coc, hblur), (double)p->max_pixel_radius * p->max_pixel_radius);
  }
  const double distance = sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
  int guarded = 1;
  if (p->sort_guard > 0.0f) { /* inSortGuard, splat form (projection.tsl.ts:145-155) */
    const double radius = fmax(fmax(sc[0], sc[1]), sc[2]) * p->max_std_dev;
    const double w = fmax(hclip[3], 1e-6);
    const double rx = e0->proj[0] * radius / w, ry = e0->proj[5] * radius / w;
    const int inside = fabs(hclip[0] / w) - rx <= (double)p->sort_guard + 1.0 &&
                       fabs(hclip[1] / w) - ry <= (double)p->sort_guard + 1.0;
    guarded = ch[2] < radius && (inside || -ch[2] <= radius);
  }
  /* headBasis (projections.tsl.ts:173-180): viewBasis, then mipInflate (projection.tsl.ts:169-197) */
  int ok = !invisible;
  double op = opacity, hq[4], hs[3];
  quat_normalize(qh, hq);
  const double smax = fmax(sc[0], fmax(sc[1], sc[2])) * 1e-4;
  for (int k = 0; k < 3; k++) hs[k] = fmax(sc[k], smax);
  {
    const double conj[4] = {-hq[0], -hq[1], -hq[2], hq[3]};
    double local[3];
    quat_rotate(conj, ch, local);
    const double l2[3] = {local[0] * local[0], local[1] * local[1], local[2] * local[2]};
    const double pixel = 2.0 / (cam->height * e0->proj[5]);
    const double footprint = pixel * pixel * (e0->ortho ? 1.0 : dot3(ch, ch));
    double s2[3], s2b[3];
    for (int k = 0; k < 3; k++) {
      s2[k] = hs[k] * hs[k] + (double)p->pre_blur_amount * footprint;
      s2b[k] = s2[k] + hblur * footprint;
    }
    const double num = l2[0] * s2[1] * s2[2] + l2[1] * s2[0] * s2[2] + l2[2] * s2[0] * s2[1];
    const double den = l2[0] * s2b[1] * s2b[2] + l2[1] * s2b[0] * s2b[2] + l2[2] * s2b[0] * s2b[1];
    op *= den > 0.0 ? sqrt(fmax(num / den, 0.0)) : 1.0;
    for (int k = 0; k < 3; k++) hs[k] = sqrt(s2b[k]);
  }
  ok = ok && op >= (double)p->min_alpha;
  int any_visible = 0;
  for (int v = 0; v < n_eyes; v++) {
    const eye_setup* e = &eyes[v];
    uint32_t ew[3] = {0u, 0u, 0u};
    double ce[3], clip[4];
    xform_point(e->from_head, ch, ce);
    clip_of(e->proj, ce, clip);
    const int cull_depth = ce[2] >= 0.0 || clip[2] < cam->ndc_z_min * clip[3] || clip[2] >= clip[3];
    if (ok && !cull_depth) {
      double eq[4];
      quat_mul(eye_q[v], hq, eq); /* frameQuat (projection.tsl.ts:101) */
      if (method == ORC_METHOD_RAYGS) {
        double fq[4], lengths[2], c2;
        if (raygs_frame(ce, e, eq, hs, std_dev, fq, lengths, &c2)) {
          const float c2f = (float)c2;
          ew[0] = orc_encode_quat_oct32(fq);
          memcpy(&ew[1], &c2f, 4);
          ew[2] = orc_encode_half(log(lengths[0])) | (orc_encode_half(log(lengths[1])) << 16);
          any_visible = 1;
        }
      } else {
        const double ndc[2] = {clip[3] > 0.0 ? clip[0] / clip[3] : 0.0, clip[3] > 0.0 ? clip[1] / clip[3] : 0.0};
        orc_bound bd = {{0.0, 0.0}, 0.0, {0.0, 0.0}};
        const int bound_ok = method == ORC_METHOD_3DGUT ? gut_bound(ce, e, eq, hs, std_dev, p, cam, &bd)
                                                        : htgs_bound(ce, ndc, e, eq, hs, std_dev, p, cam, &bd);
        const int on_screen = clip_bound_to_screen(cam, &bd);
        if (bound_ok && on_screen) {
          encode_bound(&bd, ew);
          any_visible = 1;
        }
      }
    }
    if (row)
      for (int k = 0; k < eye_words; k++) row[head_words + v * eye_words + k] = ew[k];
  }
  if (row) {
    uint32_t hw[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    if (ok) {
      uint32_t c[3];
      encode_center(ch, c);
      const double stored = op > 1.0 ? (op + 3.0) * 0.25 : op;
      hw[0] = c[0];
      hw[1] = c[1];
      hw[2] = orc_encode_ext_rgb(rgb);
      if (method == ORC_METHOD_RAYGS) {
        hw[3] = encode_opacity8(stored) | c[2];
      } else {
        hw[3] = orc_encode_quat_oct32(hq);
        hw[4] = orc_encode_half(log(hs[0])) | (orc_encode_half(log(hs[1])) << 16);
        hw[5] = orc_encode_half(log(hs[2])) | (encode_opacity8(stored) << 16) | c[2];
      }
    }
    for (int k = 0; k < head_words; k++) row[k] = hw[k];
  }
  const int keyed = cull_keys ? any_visible : (!invisible && guarded);
  if (keys) keys[gi] = keyed ? orc_sort_key(distance, sort_bits) : orc_invalid_key(sort_bits);
}

int orc_project_rays(const rdx_object* objects, int n_objects, const rdx_camera* cam, const rdx_params* params,
                     int method, int sort_bits, int cull_keys, int threads, uint32_t* words, uint32_t* keys) {
  if (cam->eyes < 1 || cam->eyes > 2) return -1;
  if (method != ORC_METHOD_3DGUT && method != ORC_METHOD_HTGS && method != ORC_METHOD_RAYGS) return -1;
  eye_setup eyes[2];
  uint64_t n = 0;
  object_setup* objs = setup_frame(objects, n_objects, cam, params, eyes, &n);
  double eye_q[2][4];
  for (int v = 0; v < cam->eyes; v++) decompose_quat(eyes[v].from_head, eye_q[v]);
  double* tq = (double*)calloc((size_t)(n_objects > 0 ? n_objects : 1) * 6, sizeof(double));
  for (int i = 0; i < n_objects; i++) tq[i * 6 + 5] = uniform_transform(objs[i].a, tq + i * 6, tq + i * 6 + 4);
#ifdef _OPENMP
  int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static, 4096) num_threads(nt)
#endif
  for (int64_t gi = 0; gi < (int64_t)n; gi++) {
    int oi = 0;
    while (oi + 1 < n_objects && (uint64_t)gi >= objs[oi + 1].offset) oi++;
    orc_splat s;
    orc_load_splat(objects[oi].table, (uint64_t)gi - objs[oi].offset, &s);
    rays_one(&s, &objs[oi], eyes, (const double(*)[4])eye_q, cam->eyes, cam, method, tq + oi * 6, tq[oi * 6 + 4],
             (int)tq[oi * 6 + 5], sort_bits, cull_keys, (uint64_t)gi, words, keys);
  }
  free(tq);
  free(objs);
  return 0;
}

/* ---- ext fixtures: src/core/splats.ts store path (encodeExt) for a raw table ---- */

/* Encoding.encodeLodOpacity, encoding.ts:209-211 */
static uint32_t encode_lod_opacity(double opacity) {
  double v = js_round(opacity * 128.0);
  return (uint32_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
}

int orc_encode_ext_table(const rdx_table* raw, uint32_t* ext_a, uint32_t* ext_b, uint32_t* const* ext_sh) {
  if (raw->layout != RDX_LAYOUT_RAW) return -1;
  const int k = SH_COEFFS[raw->sh_degree];
  for (uint64_t i = 0; i < raw->count; i++) {
    orc_splat s;
    orc_load_splat(raw, i, &s);
    uint32_t* a = ext_a + i * 4;
    uint32_t* b = ext_b + i * 4;
    for (int c = 0; c < 3; c++) {
      float f = raw->centers[i * 3 + c];
      memcpy(&a[c], &f, 4);
    }
    a[3] = encode_lod_opacity(s.opacity) << 24; /* no normal: Oct24 code 0 */
    b[0] = orc_encode_ext_rgb(s.rgb);
    b[1] = orc_encode_half(raw->log_scales[i * 3 + 0]) | (orc_encode_half(raw->log_scales[i * 3 + 1]) << 16);
    b[2] = orc_encode_half(raw->log_scales[i * 3 + 2]); /* roughness, metallic 0 */
    b[3] = orc_encode_quat_oct32(s.quat);
    for (int c = 0; c < k; c++) {
      ext_sh[c >> 2][i * 4 + (uint64_t)(c & 3)] = orc_encode_ext_rgb(&s.sh[c * 3]);
    }
    /* the padding word of a last texel is 0 */
    for (int c = k; c < ((k + 3) / 4) * 4; c++) ext_sh[c >> 2][i * 4 + (uint64_t)(c & 3)] = 0u;
  }
  return 0;
}

/* ---- gradients of the projection (raw tables) ---- */

void orc_sh_basis_grad(const double d[3], double g[24][3]) {
  const double x = d[0], y = d[1], z = d[2];
  const double xx = x * x, yy = y * y, zz = z * z;
  const double c1 = 0.4886025, c2a = 1.0925484, c2b = 0.3153916, c2c = 0.5462742;
  const double c3a = 0.5900436, c3b = 2.8906114, c3c = 0.4570458, c3d = 0.3731763, c3e = 1.4453057;
  const double c4a = 2.5033429, c4b = 1.7701308, c4c = 0.9461747, c4d = 0.6690465, c4e = 0.1057855,
               c4f = 0.4730873, c4g = 0.6258357;
  double t[24][3] = {
      {0, -c1, 0},
      {0, 0, c1},
      {-c1, 0, 0},
      {c2a * y, c2a * x, 0},
      {0, -c2a * z, -c2a * y},
      {-2 * c2b * x, -2 * c2b * y, 4 * c2b * z},
      {-c2a * z, 0, -c2a * x},
      {2 * c2c * x, -2 * c2c * y, 0},
      {-6 * c3a * x * y, -3 * c3a * (xx - yy), 0},
      {c3b * y * z, c3b * x * z, c3b * x * y},
      {2 * c3c * x * y, -c3c * (4 * zz - xx - 3 * yy), -8 * c3c * y * z},
      {-6 * c3d * x * z, -6 * c3d * y * z, c3d * (6 * zz - 3 * xx - 3 * yy)},
      {-c3c * (4 * zz - 3 * xx - yy), 2 * c3c * x * y, -8 * c3c * x * z},
      {2 * c3e * x * z, -2 * c3e * y * z, c3e * (xx - yy)},
      {-3 * c3a * (xx - yy), 6 * c3a * x * y, 0},
      {c4a * (3 * xx * y - yy * y), c4a * (xx * x - 3 * x * yy), 0},
      {-6 * c4b * x * y * z, -3 * c4b * z * (xx - yy), -c4b * y * (3 * xx - yy)},
      {c4c * y * (7 * zz - 1), c4c * x * (7 * zz - 1), 14 * c4c * x * y * z},
      {0, -c4d * z * (7 * zz - 3), -c4d * y * (21 * zz - 3)},
      {0, 0, c4e * (140 * zz * z - 60 * z)},
      {-c4d * z * (7 * zz - 3), 0, -c4d * x * (21 * zz - 3)},
      {2 * c4f * x * (7 * zz - 1), -2 * c4f * y * (7 * zz - 1), 14 * c4f * z * (xx - yy)},
      {-3 * c4b * z * (xx - yy), 6 * c4b * x * y * z, -c4b * x * (xx - 3 * yy)},
      {c4g * (4 * xx * x - 12 * x * yy), c4g * (4 * yy * y - 12 * xx * y), 0},
  };
  memcpy(g, t, sizeof(t));
}

/* m (3x3 row-major) times a vector / its transpose times a vector */
static void m3_tvec(const double m[9], const double v[3], double out[3]) {
  for (int c = 0; c < 3; c++) out[c] = m[0 * 3 + c] * v[0] + m[1 * 3 + c] * v[1] + m[2 * 3 + c] * v[2];
}

/* One visible splat's gradient: the forward of project_one in the
   covariance-matrix form, then its adjoint, summed over the eyes that draw it */
static void backward_one(const orc_splat* s, const object_setup* o, const eye_setup* eyes, int n_eyes,
                         const rdx_camera* cam, const uint8_t* vis, uint64_t gi, uint64_t n, const orc_grads_in* gin,
                         double g_center[3], double g_ls[3], double g_quat[4], double* g_opacity, double g_colors[75]) {
  const rdx_params* p = &o->params;
  memset(g_center, 0, 3 * sizeof(double));
  memset(g_ls, 0, 3 * sizeof(double));
  memset(g_quat, 0, 4 * sizeof(double));
  *g_opacity = 0.0;
  memset(g_colors, 0, 75 * sizeof(double));
  int any = 0;
  for (int v = 0; v < n_eyes; v++) any |= vis[v];
  if (!any) return;

  /* ---- forward ---- */
  double qn[4] = {s->quat[0], s->quat[1], s->quat[2], s->quat[3]};
  const double ql = sqrt(qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]);
  const int qvalid = ql > 0;
  if (qvalid) {
    for (int c = 0; c < 4; c++) qn[c] /= ql;
  } else {
    qn[0] = qn[1] = qn[2] = 0.0;
    qn[3] = 1.0;
  }
  const double qx = qn[0], qy = qn[1], qz = qn[2], qw = qn[3];
  const double R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy),
                       2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx),
                       2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)};
  double M[9], Mt[9], cov[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) M[r * 3 + c] = R[r * 3 + c] * s->scales[c];
  m3_transpose(M, Mt);
  m3_mul(M, Mt, cov);
  double a3t[9], tmp[9], acov[9];
  m3_transpose(o->a3, a3t);
  m3_mul(o->a3, cov, tmp);
  m3_mul(tmp, a3t, acov); /* A cov A^T, before the LoD inflation */
  double opacity = s->opacity, infl2 = 1.0, dop_do = 1.0;
  int op_const = 0;
  if (opacity > 1.0) {
    const double raw = opacity * 4.0 - 3.0;
    dop_do = raw < 5.0 ? 4.0 : 0.0;
    opacity = fmin(raw, 5.0);
    if (p->lod_inflate) {
      infl2 = exp(2.0 * (opacity * opacity - 1.0) / (3.0 * E_CONST));
      op_const = 1;
    }
  }
  const double op_used = op_const ? 1.0 : opacity;
  double covh[9];
  for (int k = 0; k < 9; k++) covh[k] = acov[k] * infl2;
  double ch[3];
  xform_point(o->a, s->center, ch);

  double g_covh[9] = {0}, g_ch[3] = {0}, g_op = 0.0, g_rgb[3] = {0, 0, 0};
  for (int v = 0; v < n_eyes; v++) {
    if (!vis[v]) continue;
    const eye_setup* e = &eyes[v];
    const uint64_t ei = (uint64_t)v * n + gi;
    double ce[3];
    if (e->identity) {
      memcpy(ce, ch, sizeof(ce));
    } else {
      xform_point(e->from_head, ch, ce);
    }
    double clip[4];
    clip_of(e->proj, ce, clip);
    const double ndc0 = clip[0] / clip[3], ndc1 = clip[1] / clip[3];
    double cov3[9];
    if (e->identity) {
      memcpy(cov3, covh, sizeof(cov3));
    } else {
      double ft[9], t2[9];
      m3_transpose(e->from_head3, ft);
      m3_mul(e->from_head3, covh, t2);
      m3_mul(t2, ft, cov3);
    }
    double J[9] = {0};
    const double z = ce[2];
    if (e->ortho) {
      J[0] = e->focal[0];
      J[4] = e->focal[1];
    } else {
      J[0] = e->focal[0] / z;
      J[4] = e->focal[1] / z;
      J[6] = -(e->focal[0] * ce[0]) / (z * z);
      J[7] = -(e->focal[1] * ce[1]) / (z * z);
    }
    double Jt[9], t3[9], cov2[9];
    m3_transpose(J, Jt);
    m3_mul(Jt, cov3, t3);
    m3_mul(t3, J, cov2);
    /* depth of field: blur as a function of the depth (projection.tsl.ts:117-125) */
    double blur = p->blur_amount, dblur_ddepth = 0.0;
    if (p->focal_distance > 0.0f && p->aperture_tan > 0.0f && z < 0.0) {
      const double depth = -z;
      const double fp = cam->height * 0.5 * e->proj[5];
      const double dist = depth - (double)p->focal_distance;
      const double coc_view = fabs(dist) * (double)p->aperture_tan;
      const double coc = e->ortho ? coc_view * fp : coc_view * fp / depth;
      const double dcoc = e->ortho ? (dist >= 0 ? 1.0 : -1.0) * p->aperture_tan * fp
                                   : ((dist >= 0 ? 1.0 : -1.0) * p->aperture_tan * fp / depth - coc / depth);
      const double maxr2 = (double)p->max_pixel_radius * p->max_pixel_radius;
      const double c2 = coc * coc;
      if (c2 > blur && c2 < maxr2) dblur_ddepth = 2.0 * coc * dcoc;
      blur = fmin(fmax(c2, blur), maxr2);
    }
    const double pre = p->pre_blur_amount;
    const double a0 = cov2[0] + pre, d0 = cov2[4] + pre, b = cov2[1];
    const double det_orig = a0 * d0 - b * b;
    const double a = a0 + blur, d = d0 + blur;
    const double det = a * d - b * b;
    const double r = det_orig / det;

    /* ---- adjoint ---- */
    const double gm0 = gin->mean2d ? gin->mean2d[ei * 2] : 0.0, gm1 = gin->mean2d ? gin->mean2d[ei * 2 + 1] : 0.0;
    const double gc0 = gin->conic ? gin->conic[ei * 3] : 0.0, gc1 = gin->conic ? gin->conic[ei * 3 + 1] : 0.0,
                 gc2 = gin->conic ? gin->conic[ei * 3 + 2] : 0.0;
    const double gd = gin->depth ? gin->depth[ei] : 0.0;
    const double go = gin->opacity ? gin->opacity[ei] : 0.0;
    if (gin->rgb)
      for (int c = 0; c < 3; c++) g_rgb[c] += gin->rgb[ei * 3 + c];
    /* conic = (d, -b, a) / det */
    double G_a = gc2 / det, G_d = gc0 / det, G_b = -gc1 / det;
    double G_det = (-gc0 * d + gc1 * b - gc2 * a) / (det * det);
    /* opacity = op sqrt(det_orig / det) */
    double G_det_orig = 0.0;
    if (r > 0.0) {
      const double sr = sqrt(r);
      g_op += go * sr;
      const double G_r = go * op_used / (2.0 * sr);
      G_det_orig = G_r / det;
      G_det += -G_r * r / det;
    }
    G_a += G_det * d;
    G_d += G_det * a;
    G_b += -2.0 * b * G_det;
    const double G_a0 = G_a + G_det_orig * d0, G_d0 = G_d + G_det_orig * a0;
    G_b += -2.0 * b * G_det_orig;
    const double G_blur = G_a + G_d;
    /* cov2 = J^T cov3 J, read at [0], [1] and [4] */
    double G2[9] = {0};
    G2[0] = G_a0;
    G2[1] = G_b;
    G2[4] = G_d0;
    double G2s[9], JG[9], g_cov3[9], tmpg[9];
    for (int k = 0; k < 9; k++) G2s[k] = G2[k] + G2[(k % 3) * 3 + k / 3]; /* G2 + G2^T */
    m3_mul(J, G2, JG);
    m3_mul(JG, Jt, g_cov3); /* J G2 J^T */
    double CJ[9], g_J[9];
    m3_mul(cov3, J, tmpg);
    memcpy(CJ, tmpg, sizeof(CJ));
    m3_mul(CJ, G2s, g_J); /* cov3 J (G2 + G2^T) */
    double g_ce[3] = {0, 0, 0};
    if (!e->ortho) {
      const double fx = e->focal[0], fy = e->focal[1];
      g_ce[0] += g_J[6] * (-fx / (z * z));
      g_ce[1] += g_J[7] * (-fy / (z * z));
      g_ce[2] += g_J[0] * (-fx / (z * z)) + g_J[4] * (-fy / (z * z)) + g_J[6] * (2.0 * fx * ce[0] / (z * z * z)) +
                 g_J[7] * (2.0 * fy * ce[1] / (z * z * z));
    }
    g_ce[2] += -G_blur * dblur_ddepth; /* depth = -z */
    /* mean2d = (ndc + 1) / 2 * size, ndc = clip.xy / clip.w */
    const double g_n0 = gm0 * 0.5 * cam->width, g_n1 = gm1 * 0.5 * cam->height;
    const double g_cl[4] = {g_n0 / clip[3], g_n1 / clip[3], 0.0, -(g_n0 * ndc0 + g_n1 * ndc1) / clip[3]};
    for (int c = 0; c < 3; c++)
      for (int rr = 0; rr < 4; rr++) g_ce[c] += e->proj[c * 4 + rr] * g_cl[rr];
    g_ce[2] += -gd;
    /* cov3 = F covh F^T, ce = F ch + f */
    if (e->identity) {
      for (int k = 0; k < 9; k++) g_covh[k] += g_cov3[k];
      for (int c = 0; c < 3; c++) g_ch[c] += g_ce[c];
    } else {
      double ft[9], t4[9], t5[9], gh[3];
      m3_transpose(e->from_head3, ft);
      m3_mul(ft, g_cov3, t4);
      m3_mul(t4, e->from_head3, t5);
      for (int k = 0; k < 9; k++) g_covh[k] += t5[k];
      m3_tvec(e->from_head3, g_ce, gh);
      for (int c = 0; c < 3; c++) g_ch[c] += gh[c];
    }
  }
  /* ch = A c + t */
  double gc_[3];
  m3_tvec(o->a3, g_ch, gc_);
  for (int c = 0; c < 3; c++) g_center[c] += gc_[c];
  /* covh = infl2 A cov A^T */
  double g_infl2 = 0.0;
  for (int k = 0; k < 9; k++) g_infl2 += g_covh[k] * acov[k];
  double t6[9], t7[9], g_cov[9];
  m3_mul(a3t, g_covh, t6);
  m3_mul(t6, o->a3, t7);
  for (int k = 0; k < 9; k++) g_cov[k] = t7[k] * infl2;
  /* cov = M M^T: g_M = (g_cov + g_cov^T) M */
  double gcs[9], g_M[9];
  for (int k = 0; k < 9; k++) gcs[k] = g_cov[k] + g_cov[(k % 3) * 3 + k / 3];
  m3_mul(gcs, M, g_M);
  double g_R[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      g_R[r * 3 + c] = g_M[r * 3 + c] * s->scales[c];
      g_ls[c] += g_M[r * 3 + c] * R[r * 3 + c] * s->scales[c]; /* d s / d ln s = s */
    }
  /* R(q) of the normalised quaternion, then the normalisation */
  if (qvalid) {
    const double* G = g_R;
    double gq[4];
    gq[0] = G[1] * 2 * qy + G[2] * 2 * qz + G[3] * 2 * qy + G[4] * -4 * qx + G[5] * -2 * qw + G[6] * 2 * qz +
            G[7] * 2 * qw + G[8] * -4 * qx;
    gq[1] = G[0] * -4 * qy + G[1] * 2 * qx + G[2] * 2 * qw + G[3] * 2 * qx + G[5] * 2 * qz + G[6] * -2 * qw +
            G[7] * 2 * qz + G[8] * -4 * qy;
    gq[2] = G[0] * -4 * qz + G[1] * -2 * qw + G[2] * 2 * qx + G[3] * 2 * qw + G[4] * -4 * qz + G[5] * 2 * qy +
            G[6] * 2 * qx + G[7] * 2 * qy;
    gq[3] = G[1] * -2 * qz + G[2] * 2 * qy + G[3] * 2 * qz + G[5] * -2 * qx + G[6] * -2 * qy + G[7] * 2 * qx;
    const double dotq = gq[0] * qx + gq[1] * qy + gq[2] * qz + gq[3] * qw;
    for (int c = 0; c < 4; c++) g_quat[c] = (gq[c] - qn[c] * dotq) / ql;
  }
  /* opacity: the LoD stretch and inflation (projection.tsl.ts:42-64) */
  if (op_const) {
    const double g_opl = g_infl2 * infl2 * 4.0 * opacity / (3.0 * E_CONST);
    *g_opacity = g_opl * dop_do;
  } else {
    *g_opacity = g_op * dop_do;
  }
  /* colour: rgb = max(base + SH, 0) with SH (GpuShReader.apply), base alone without */
  const int degree = s->sh_degree < p->max_sh_degree ? s->sh_degree : p->max_sh_degree;
  if (s->sh_degree < 1) {
    for (int c = 0; c < 3; c++) g_colors[c] = g_rgb[c];
    return;
  }
  double sh[3] = {0, 0, 0}, dir[3] = {0, 0, 0}, len = 0.0;
  double dv[3] = {s->center[0] - o->origin[0], s->center[1] - o->origin[1], s->center[2] - o->origin[2]};
  if (degree >= 1) {
    len = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    if (len > 0)
      for (int c = 0; c < 3; c++) dir[c] = dv[c] / len;
    orc_sh_evaluate(s->sh, dir, degree, sh);
  }
  double gm[3];
  for (int c = 0; c < 3; c++) {
    gm[c] = s->rgb[c] + sh[c] > 0.0 ? g_rgb[c] : 0.0;
    g_colors[c] = gm[c];
  }
  if (degree >= 1 && len > 0) {
    double basis[24], db[24][3], g_dir[3] = {0, 0, 0};
    orc_sh_basis(dir, basis);
    orc_sh_basis_grad(dir, db);
    for (int k = 0; k < SH_COEFFS[degree]; k++) {
      for (int c = 0; c < 3; c++) {
        g_colors[3 + k * 3 + c] = gm[c] * basis[k];
        for (int j = 0; j < 3; j++) g_dir[j] += gm[c] * s->sh[k * 3 + c] * db[k][j];
      }
    }
    const double dd = g_dir[0] * dir[0] + g_dir[1] * dir[1] + g_dir[2] * dir[2];
    for (int j = 0; j < 3; j++) g_center[j] += (g_dir[j] - dir[j] * dd) / len;
  }
}

int orc_project_backward(const rdx_object* objects, int n_objects, const rdx_camera* cam, const rdx_params* params,
                         const orc_grads_in* gin, const orc_grads_out* gout, int threads) {
  if (cam->eyes < 1 || cam->eyes > 2) return -1;
  for (int i = 0; i < n_objects; i++)
    if (objects[i].table->layout != RDX_LAYOUT_RAW) return -1;
  eye_setup eyes[2];
  uint64_t n = 0;
  object_setup* objs = setup_frame(objects, n_objects, cam, params, eyes, &n);
#ifdef _OPENMP
  int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static, 1024) num_threads(nt)
#endif
  for (int64_t gi = 0; gi < (int64_t)n; gi++) {
    int oi = 0;
    while (oi + 1 < n_objects && (uint64_t)gi >= objs[oi + 1].offset) oi++;
    orc_splat s;
    orc_load_splat(objects[oi].table, (uint64_t)gi - objs[oi].offset, &s);
    /* the forward's cull decisions, per eye */
    uint8_t vis[2] = {0, 0};
    orc_outputs one;
    memset(&one, 0, sizeof(one));
    one.visible = vis;
    project_one(&s, &objs[oi], eyes, cam->eyes, cam, 32, 1, 0, 1, &one);
    double gcen[3], gls[3], gq[4], gop, gcol[75];
    backward_one(&s, &objs[oi], eyes, cam->eyes, cam, vis, (uint64_t)gi, n, gin, gcen, gls, gq, &gop, gcol);
    if (gout->centers) memcpy(gout->centers + gi * 3, gcen, sizeof(gcen));
    if (gout->log_scales) memcpy(gout->log_scales + gi * 3, gls, sizeof(gls));
    if (gout->quats) memcpy(gout->quats + gi * 4, gq, sizeof(gq));
    if (gout->opacities) gout->opacities[gi] = gop;
    if (gout->colors) memcpy(gout->colors + gi * 75, gcol, sizeof(gcol));
  }
  free(objs);
  return 0;
}

/* ---- fixtures of the packed and cov layouts and of the SH codecs ---- */

/* packedCodec.encode (splats.ts:279-286) of a raw table */
int orc_encode_packed_table(const rdx_table* raw, const float encoding[4], uint32_t* packed) {
  if (raw->layout != RDX_LAYOUT_RAW) return -1;
  const double rmin = encoding[0], rmax = encoding[1], lmin = encoding[2], lmax = encoding[3];
  const double range = rmax - rmin, step = (lmax - lmin) / 254.0;
  for (uint64_t i = 0; i < raw->count; i++) {
    orc_splat s;
    orc_load_splat(raw, i, &s);
    uint32_t* p = packed + i * 4;
    uint32_t rgb = 0;
    for (int c = 0; c < 3; c++) rgb |= encode_unorm8((s.rgb[c] - rmin) / range) << (8 * c);
    const uint32_t quat = orc_encode_quat_oct(s.quat, 8, 8);
    p[0] = rgb | (encode_unorm8(s.opacity) << 24);
    p[1] = orc_encode_half(s.center[0]) | (orc_encode_half(s.center[1]) << 16);
    p[2] = orc_encode_half(s.center[2]) | ((quat & 0xffffu) << 16);
    uint32_t w = 0;
    for (int c = 0; c < 3; c++) {
      const double v = s.scales[c];
      uint32_t code = 0;
      if (v > 0) {
        double r = js_round((log(v) - lmin) / step) + 1.0;
        code = (uint32_t)(r < 1 ? 1 : (r > 255 ? 255 : r));
      }
      w |= code << (8 * c);
    }
    p[3] = w | ((quat >> 16) << 24);
  }
  return 0;
}

static double encode_correlation(double value, double a, double b) { /* splats.ts:223-229 */
  double c = value / sqrt(a * b);
  c = c < -1 ? -1 : (c > 1 ? 1 : c);
  if (c == 0 || !isfinite(c)) return 0.0;
  double l = log(fabs(c));
  l = l < -100 ? -100 : (l > -1e-7 ? -1e-7 : l);
  return (c > 0 ? 1.0 : -1.0) * l;
}

/* storeCovFields (splats.ts:236-243) of a raw table: the covariance of its
   scales and rotation, the base rgb and the LoD opacity byte */
int orc_encode_cov_table(const rdx_table* raw, uint32_t* cov_a, uint32_t* cov_b) {
  if (raw->layout != RDX_LAYOUT_RAW) return -1;
  for (uint64_t i = 0; i < raw->count; i++) {
    orc_splat s;
    orc_load_splat(raw, i, &s);
    double qx = s.quat[0], qy = s.quat[1], qz = s.quat[2], qw = s.quat[3];
    double ql = sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
    if (ql > 0) {
      qx /= ql;
      qy /= ql;
      qz /= ql;
      qw /= ql;
    } else {
      qx = qy = qz = 0;
      qw = 1;
    }
    const double sx = s.scales[0], sy = s.scales[1], sz = s.scales[2];
    const double M[9] = {
        sx * (1 - 2 * (qy * qy + qz * qz)), sy * 2 * (qx * qy - qw * qz), sz * 2 * (qx * qz + qw * qy),
        sx * 2 * (qx * qy + qw * qz), sy * (1 - 2 * (qx * qx + qz * qz)), sz * 2 * (qy * qz - qw * qx),
        sx * 2 * (qx * qz - qw * qy), sy * 2 * (qy * qz + qw * qx), sz * (1 - 2 * (qx * qx + qy * qy)),
    };
    double Mt[9], cov[9];
    m3_transpose(M, Mt);
    m3_mul(M, Mt, cov);
    const double xx = cov[0], yy = cov[4], zz = cov[8];
    uint32_t* a = cov_a + i * 4;
    uint32_t* b = cov_b + i * 4;
    for (int c = 0; c < 3; c++) {
      float f = (float)s.center[c];
      memcpy(&a[c], &f, 4);
    }
    a[3] = encode_lod_opacity(s.opacity) << 24;
    b[0] = orc_encode_ext_rgb(s.rgb);
    b[1] = orc_encode_half(log(xx)) | (orc_encode_half(log(yy)) << 16);
    b[2] = orc_encode_half(log(zz)) | (orc_encode_half(encode_correlation(cov[1], xx, yy)) << 16);
    b[3] = orc_encode_half(encode_correlation(cov[2], xx, zz)) | (orc_encode_half(encode_correlation(cov[5], yy, zz)) << 16);
  }
  return 0;
}

int orc_sh_words(int codec, int degree) {
  static const int PACKED_BYTES[5] = {0, 10, 26, 48, 76};
  if (degree < 0 || degree > 4) return 0;
  return codec == RDX_SH_PACKED ? (PACKED_BYTES[degree] + 3) / 4 : SH_COEFFS[degree];
}

/* The codec words of a raw table's SH coefficients (sh.ts:137-160), [count][stride] */
int orc_encode_sh(const rdx_table* raw, int codec, uint32_t* words, int stride) {
  if (raw->layout != RDX_LAYOUT_RAW) return -1;
  const int deg = raw->sh_degree;
  if (stride < orc_sh_words(codec, deg)) return -1;
  for (uint64_t i = 0; i < raw->count; i++) {
    orc_splat s;
    orc_load_splat(raw, i, &s);
    uint32_t* out = words + i * (uint64_t)stride;
    memset(out, 0, (size_t)stride * 4);
    if (codec == RDX_SH_PACKED) {
      int byte = 0;
      for (int band = 0; band < deg; band++) {
        const int first = SH_COEFFS[band] * 3, end = SH_COEFFS[band + 1] * 3;
        double max = 0.0;
        for (int v = first; v < end; v++) max = fmax(max, fabs(s.sh[v]));
        const uint32_t code = encode_sh_scale(max);
        const double scale = decode_sh_scale(code);
        out[byte >> 2] |= code << ((byte & 3) * 8);
        for (int v = first; v < end; v++) {
          int b = byte + 1 + v - first;
          double q = scale > 0 ? js_round(s.sh[v] / scale * 127.0) : 0.0;
          int32_t qi = (int32_t)(q < -127 ? -127 : (q > 127 ? 127 : q));
          out[b >> 2] |= ((uint32_t)qi & 0xffu) << ((b & 3) * 8);
        }
        byte += PACKED_BAND_BYTES[band];
      }
    } else {
      for (int c = 0; c < SH_COEFFS[deg]; c++) out[c] = orc_encode_ext_rgb(&s.sh[c * 3]);
    }
  }
  return 0;
}

/* ---- PLY files: PlyFile.read (src/core/ply.ts:58-264) in float64 ---- */

typedef struct ply_prop {
  char name[64];
  int type; /* 0 char .. 7 double, -1 list */
  int offset;
} ply_prop;

typedef struct ply_elem {
  char name[64];
  uint64_t count;
  int n_props;
  ply_prop props[256];
  int record;
} ply_elem;

static const int PLY_BYTES[8] = {1, 1, 2, 2, 4, 4, 4, 8};
static const double PLY_SCALE[8] = {127, 255, 32767, 65535, 2147483647.0, 4294967295.0, 1, 1}; /* ply.ts:33-42 */

static int ply_type_of(const char* s) { /* ply.ts:413-423 */
  static const char* names[8] = {"char", "uchar", "short", "ushort", "int", "uint", "float", "double"};
  static const char* aliases[8] = {"int8", "uint8", "int16", "uint16", "int32", "uint32", "float32", "float64"};
  for (int t = 0; t < 8; t++)
    if (!strcmp(s, names[t]) || !strcmp(s, aliases[t])) return t;
  return -2;
}

static const ply_prop* ply_find(const ply_elem* e, const char* name) {
  for (int i = 0; i < e->n_props; i++)
    if (e->props[i].type >= 0 && !strcmp(e->props[i].name, name)) return &e->props[i];
  return NULL;
}

static double ply_read(const uint8_t* rec, const ply_prop* p, int little, int normalized) { /* ply.ts:446-469 */
  const uint8_t* at = rec + p->offset;
  const int n = PLY_BYTES[p->type];
  uint64_t bits = 0;
  for (int b = 0; b < n; b++) bits |= (uint64_t)at[b] << (8 * (little ? b : n - 1 - b));
  double v;
  switch (p->type) {
    case 0: v = (double)(int8_t)bits; break;
    case 1: v = (double)(uint8_t)bits; break;
    case 2: v = (double)(int16_t)bits; break;
    case 3: v = (double)(uint16_t)bits; break;
    case 4: v = (double)(int32_t)bits; break;
    case 5: v = (double)(uint32_t)bits; break;
    case 6: {
      uint32_t u = (uint32_t)bits;
      float f;
      memcpy(&f, &u, 4);
      v = f;
      break;
    }
    default: {
      double dd;
      memcpy(&dd, &bits, 8);
      v = dd;
    }
  }
  return normalized ? v / PLY_SCALE[p->type] : v;
}

static int ply_degree(int rest) { return rest >= 72 ? 4 : rest >= 45 ? 3 : rest >= 24 ? 2 : rest > 0 ? 1 : 0; }

int orc_ply_decode(const uint8_t* bytes, uint64_t nbytes, int sh_degree, double* centers, double* log_scales,
                   double* quats, double* opacities, double* colors, uint64_t* count_out, int* degree_out,
                   int* kind_out) {
  const uint64_t head = nbytes < 65536 ? nbytes : 65536;
  if (head < 3 || memcmp(bytes, "ply", 3) != 0) return -1;
  /* the header lines up to end_header */
  uint64_t pos = 0, header_len = 0;
  int little = -1;
  static ply_elem elems[16];
  int n_elems = 0;
  char line[512];
  while (pos < head) {
    uint64_t e = pos;
    while (e < head && bytes[e] != '\n') e++;
    if (e >= head) return -1;
    uint64_t len = e - pos;
    if (len && bytes[e - 1] == '\r') len--;
    if (len >= sizeof(line)) len = sizeof(line) - 1;
    memcpy(line, bytes + pos, len);
    line[len] = 0;
    pos = e + 1;
    if (!strcmp(line, "end_header")) {
      header_len = pos;
      break;
    }
    char f0[64] = "", f1[64] = "", f2[64] = "", f3[64] = "", f4[64] = "";
    int nf = sscanf(line, "%63s %63s %63s %63s %63s", f0, f1, f2, f3, f4);
    if (nf <= 0) continue;
    if (!strcmp(f0, "format")) {
      if (!strcmp(f1, "binary_little_endian")) little = 1;
      else if (!strcmp(f1, "binary_big_endian")) little = 0;
      else return -1;
    } else if (!strcmp(f0, "element") && nf >= 3 && n_elems < 16) {
      ply_elem* el = &elems[n_elems++];
      memset(el, 0, sizeof(*el));
      snprintf(el->name, sizeof(el->name), "%s", f1);
      el->count = strtoull(f2, NULL, 10);
    } else if (!strcmp(f0, "property") && n_elems > 0) {
      ply_elem* el = &elems[n_elems - 1];
      if (el->n_props >= 256) return -1;
      ply_prop* p = &el->props[el->n_props++];
      if (!strcmp(f1, "list")) {
        snprintf(p->name, sizeof(p->name), "%s", f4);
        p->type = -1;
        p->offset = -1;
      } else {
        snprintf(p->name, sizeof(p->name), "%s", f2);
        p->type = ply_type_of(f1);
        if (p->type < 0) return -1;
        p->offset = el->record;
        el->record += PLY_BYTES[p->type];
      }
    }
  }
  if (!header_len || little < 0) return -1;
  const ply_elem *vertex = NULL, *chunk = NULL, *sh = NULL;
  uint64_t offs[16], off = header_len;
  for (int i = 0; i < n_elems; i++) {
    offs[i] = off;
    off += elems[i].count * (uint64_t)elems[i].record;
    if (!strcmp(elems[i].name, "vertex") && !vertex) vertex = &elems[i];
    if (!strcmp(elems[i].name, "chunk") && !chunk) chunk = &elems[i];
    if (!strcmp(elems[i].name, "sh") && !sh) sh = &elems[i];
  }
  if (!vertex) return -1;
  const uint64_t vo = offs[vertex - elems];
  if (vo + vertex->count * (uint64_t)vertex->record > nbytes) return -1;
  const uint64_t n = vertex->count;
  *count_out = n;
  char name[64];
  static const char* packed_names[4] = {"packed_position", "packed_rotation", "packed_scale", "packed_color"};
  int compressed = chunk != NULL;
  for (int k = 0; k < 4 && compressed; k++) compressed = ply_find(vertex, packed_names[k]) != NULL;
  int degree = 0, rest = 0;
  if (compressed) {
    if (sh)
      for (;;) {
        snprintf(name, sizeof(name), "f_rest_%d", rest);
        if (!ply_find(sh, name)) break;
        rest++;
      }
    degree = (sh && sh->count >= n) ? ply_degree(rest) : 0;
    *kind_out = 2;
  } else {
    for (;;) {
      snprintf(name, sizeof(name), "f_rest_%d", rest);
      if (!ply_find(vertex, name)) break;
      rest++;
    }
    *kind_out = ply_find(vertex, "scale_0") ? 0 : 1;
    degree = *kind_out == 0 ? ply_degree(rest) : 0;
  }
  *degree_out = degree;
  if (sh_degree < 0) sh_degree = degree;
  if (sh_degree > degree) return -1;
  const int kvals = SH_COEFFS[sh_degree] * 3, row = 3 + kvals, per = rest / 3;
  for (uint64_t i = 0; i < n; i++) {
    const uint8_t* v = bytes + vo + i * (uint64_t)vertex->record;
    double c[3], ls[3], q[4], op, rgb[3];
    double* col = colors ? colors + i * (uint64_t)row : NULL;
    if (compressed) { /* ply.ts:222-262 */
      static const char* cn[18] = {"min_x", "min_y", "min_z", "max_x", "max_y", "max_z",
                                   "min_scale_x", "min_scale_y", "min_scale_z", "max_scale_x", "max_scale_y", "max_scale_z",
                                   "min_r", "min_g", "min_b", "max_r", "max_g", "max_b"};
      const double defaults[6] = {0, 0, 0, 1, 1, 1};
      const uint8_t* ch = bytes + offs[chunk - elems] + (i / 256) * (uint64_t)chunk->record;
      double r[18];
      for (int k = 0; k < 18; k++) {
        const ply_prop* p = ply_find(chunk, cn[k]);
        r[k] = p ? ply_read(ch, p, little, 0) : defaults[k >= 12 ? k - 12 : 0];
      }
      uint32_t words[4];
      for (int k = 0; k < 4; k++) words[k] = (uint32_t)ply_read(v, ply_find(vertex, packed_names[k]), little, 0);
      const uint32_t pw = words[0], rw = words[1], lw = words[2], kw = words[3];
      c[0] = r[0] + (r[3] - r[0]) * ((double)((pw >> 21) & 2047) / 2047);
      c[1] = r[1] + (r[4] - r[1]) * ((double)((pw >> 11) & 1023) / 1023);
      c[2] = r[2] + (r[5] - r[2]) * ((double)(pw & 2047) / 2047);
      ls[0] = r[6] + (r[9] - r[6]) * ((double)((lw >> 21) & 2047) / 2047);
      ls[1] = r[7] + (r[10] - r[7]) * ((double)((lw >> 11) & 1023) / 1023);
      ls[2] = r[8] + (r[11] - r[8]) * ((double)(lw & 2047) / 2047);
      const double a = ((double)((rw >> 20) & 1023) / 1023 - 0.5) * sqrt(2.0);
      const double b = ((double)((rw >> 10) & 1023) / 1023 - 0.5) * sqrt(2.0);
      const double cc = ((double)(rw & 1023) / 1023 - 0.5) * sqrt(2.0);
      const double m = sqrt(fmax(0.0, 1 - a * a - b * b - cc * cc));
      const uint32_t largest = rw >> 30;
      q[3] = largest == 0 ? m : a;
      q[0] = largest == 0 ? a : largest == 1 ? m : b;
      q[1] = largest <= 1 ? b : largest == 2 ? m : cc;
      q[2] = largest <= 2 ? cc : m;
      rgb[0] = r[12] + (r[15] - r[12]) * ((double)((kw >> 24) & 255) / 255);
      rgb[1] = r[13] + (r[16] - r[13]) * ((double)((kw >> 16) & 255) / 255);
      rgb[2] = r[14] + (r[17] - r[14]) * ((double)((kw >> 8) & 255) / 255);
      op = (double)(kw & 255) / 255;
      if (col) {
        const uint8_t* srec = (sh && degree > 0) ? bytes + offs[sh - elems] + i * (uint64_t)sh->record : NULL;
        for (int x = 0; x < kvals; x++) {
          double val = 0.0;
          if (srec) {
            snprintf(name, sizeof(name), "f_rest_%d", (x % 3) * per + x / 3);
            const ply_prop* p = ply_find(sh, name);
            const uint32_t byte = srec[p ? p->offset : 0];
            val = ((byte == 0 ? 0 : byte == 255 ? 1 : (byte + 0.5) / 256) - 0.5) * 8; /* ply.ts:267-270 */
          }
          col[3 + x] = val;
        }
      }
    } else {
      c[0] = ply_read(v, ply_find(vertex, "x"), little, 0);
      c[1] = ply_read(v, ply_find(vertex, "y"), little, 0);
      c[2] = ply_read(v, ply_find(vertex, "z"), little, 0);
      if (*kind_out == 0) { /* ply.ts:129-146 */
        for (int k = 0; k < 3; k++) {
          snprintf(name, sizeof(name), "scale_%d", k);
          ls[k] = ply_read(v, ply_find(vertex, name), little, 0);
        }
        q[0] = ply_read(v, ply_find(vertex, "rot_1"), little, 0);
        q[1] = ply_read(v, ply_find(vertex, "rot_2"), little, 0);
        q[2] = ply_read(v, ply_find(vertex, "rot_3"), little, 0);
        q[3] = ply_read(v, ply_find(vertex, "rot_0"), little, 0);
        op = 1.0 / (1.0 + exp(-ply_read(v, ply_find(vertex, "opacity"), little, 0)));
        for (int k = 0; k < 3; k++) {
          snprintf(name, sizeof(name), "f_dc_%d", k);
          rgb[k] = 0.5 + 0.28209479177387814 * ply_read(v, ply_find(vertex, name), little, 0);
        }
        if (col)
          for (int x = 0; x < kvals; x++) {
            snprintf(name, sizeof(name), "f_rest_%d", (x % 3) * per + x / 3);
            col[3 + x] = ply_read(v, ply_find(vertex, name), little, 0);
          }
      } else { /* a point cloud: ply.ts:147-155 */
        ls[0] = ls[1] = ls[2] = log(0.001);
        q[0] = q[1] = q[2] = 0;
        q[3] = 1;
        const ply_prop* alpha = ply_find(vertex, "alpha");
        op = alpha ? ply_read(v, alpha, little, 1) : 1.0;
        rgb[0] = ply_read(v, ply_find(vertex, "red"), little, 1);
        rgb[1] = ply_read(v, ply_find(vertex, "green"), little, 1);
        rgb[2] = ply_read(v, ply_find(vertex, "blue"), little, 1);
        if (col)
          for (int x = 0; x < kvals; x++) col[3 + x] = 0.0;
      }
    }
    const double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]); /* math.ts:12-27 */
    if (len > 0) {
      for (int k = 0; k < 4; k++) q[k] /= len;
    } else {
      q[0] = q[1] = q[2] = 0;
      q[3] = 1;
    }
    if (centers) memcpy(centers + i * 3, c, sizeof(c));
    if (log_scales) memcpy(log_scales + i * 3, ls, sizeof(ls));
    if (quats) memcpy(quats + i * 4, q, sizeof(q));
    if (opacities) opacities[i] = op;
    if (col) memcpy(col, rgb, sizeof(rgb));
  }
  return 0;
}

/* ---- SPZ: src/core/spz.ts:285-348 (per splat), 571-586 (smallest three) ---- */

static const int SPZ_SH_VECTORS[5] = {0, 3, 8, 15, 24};

/* decodeSmallestThree: the largest component's index in the top 2 bits, then
   the other three from the highest index down, 10 bits each (sign bit 9,
   magnitude over sqrt(1/2) in bits 0-8) from the low bits up */
static void spz_smallest_three(uint32_t packed, double q[4]) {
  const int largest = (int)(packed >> 30);
  uint32_t rest = packed;
  double sum = 0.0;
  for (int i = 3; i >= 0; i--) {
    if (i == largest) continue;
    const double mag = (double)(rest & 511u) / 511.0;
    const double v = 0.7071067811865476 * mag * ((rest >> 9) & 1u ? -1.0 : 1.0);
    rest >>= 10;
    q[i] = v;
    sum += v * v;
  }
  q[largest] = sqrt(fmax(1.0 - sum, 0.0));
}

int orc_spz_decode(int version, uint64_t count, int sh_degree, int fractional_bits, const uint8_t* centers,
                   const uint8_t* alphas, const uint8_t* colors, const uint8_t* scales, const uint8_t* rotations,
                   const uint8_t* sh, int out_degree, double* out_centers, double* out_log_scales, double* out_quats,
                   double* out_opacities, double* out_colors) {
  if (version < 1 || version > 4 || sh_degree < 0 || sh_degree > 4 || out_degree < 0 || out_degree > sh_degree)
    return -1;
  const double color_scale = 0.28209479177387814 / 0.15;
  /* fixed = 1 / (1 << fractionalBits) with a 32-bit shift, as JS evaluates it */
  const int32_t unit = (int32_t)(1u << (fractional_bits & 31));
  const double fixed = 1.0 / (double)unit;
  const int file_k = SPZ_SH_VECTORS[sh_degree], out_k = SPZ_SH_VECTORS[out_degree];
  for (uint64_t i = 0; i < count; i++) {
    if (out_centers) {
      for (int c = 0; c < 3; c++) {
        double v;
        if (version == 1) {
          const uint8_t* p = centers + i * 6 + c * 2;
          v = orc_decode_half((uint32_t)p[0] | ((uint32_t)p[1] << 8));
        } else {
          const uint8_t* p = centers + i * 9 + c * 3;
          int32_t code = (int32_t)((uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16));
          if (code & 0x800000) code -= 0x1000000;
          v = (double)code * fixed;
        }
        out_centers[i * 3 + c] = v;
      }
    }
    if (out_opacities) out_opacities[i] = (double)alphas[i] / 255.0;
    if (out_log_scales)
      for (int c = 0; c < 3; c++) out_log_scales[i * 3 + c] = (double)scales[i * 3 + c] / 16.0 - 10.0;
    if (out_quats) {
      double q[4];
      if (version >= 3) {
        const uint8_t* p = rotations + i * 4;
        spz_smallest_three((uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24), q);
      } else {
        const uint8_t* p = rotations + i * 3;
        q[0] = (double)p[0] / 127.5 - 1.0;
        q[1] = (double)p[1] / 127.5 - 1.0;
        q[2] = (double)p[2] / 127.5 - 1.0;
        q[3] = sqrt(fmax(0.0, 1.0 - q[0] * q[0] - q[1] * q[1] - q[2] * q[2]));
      }
      /* the raw table's quaternions are normalised */
      const double l2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
      const double inv = l2 > 0.0 ? 1.0 / sqrt(l2) : 0.0;
      for (int c = 0; c < 4; c++) out_quats[i * 4 + c] = l2 > 0.0 ? q[c] * inv : (c == 3 ? 1.0 : 0.0);
    }
    if (out_colors) {
      double* row = out_colors + i * (size_t)(1 + out_k) * 3;
      for (int c = 0; c < 3; c++) row[c] = ((double)colors[i * 3 + c] / 255.0 - 0.5) * color_scale + 0.5;
      for (int k = 0; k < out_k; k++)
        for (int c = 0; c < 3; c++) row[3 + k * 3 + c] = ((double)sh[(i * file_k + k) * 3 + c] - 128.0) / 128.0;
    }
  }
  return 0;
}
