// The ray projection methods for sm_100a: 3dgut, htgs and raygs words and the
// sort key of every splat, one thread per splat.
//
// Restates rayProjection with gutBound / htgsBound and raygs
// (src/render/projections.tsl.ts:170-474), headBasis / viewBasis / mipInflate,
// the bounds and their codecs (src/render/projection.tsl.ts:167-366),
// transformUniform and transformSplat (src/render/splatTransform.tsl.ts:
// 117-162), fromCov with symEigens (src/gpu/splats.tsl.ts:189-199,
// src/gpu/math.tsl.ts:46-112) and SplatProjection.project / write
// (src/render/SplatProjection.ts:126-153).
//
// A row holds H head words, then W words per eye (H, W = 6, 2 for 3dgut and
// htgs; 4, 3 for raygs), in the reference's word order. A culled eye's words
// are zero; the head words are zero when the head basis drops the splat
// (invisible, or its MIP-compensated opacity below minAlpha).
//
// Precision: float64 throughout, rounded once into the words. This file is
// compiled without contraction of multiplies and adds (--fmad=false), so
// every arithmetic step rounds as the float64 CPU oracle's does; only the
// library's transcendental functions (exp, log, log2, pow, sin, cos, atan2,
// acos) may differ from the host's by an ulp. The head-space centre, the key
// distance and the depth cull therefore equal the oracle's, and with them
// the keys.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"
#include "table_rows.cuh"

namespace rdx {
namespace {

constexpr int kRayWarps = 4;  // warps per block; a warp takes a 32-splat tile

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// quatRotate (src/gpu/math.tsl.ts:12-15): v + w t + q.xyz x t with t = 2 q.xyz x v
__device__ __forceinline__ void quat_rotate(const double q[4], const double v[3], double out[3]) {
  const double t0 = 2.0 * (q[1] * v[2] - q[2] * v[1]), t1 = 2.0 * (q[2] * v[0] - q[0] * v[2]),
               t2 = 2.0 * (q[0] * v[1] - q[1] * v[0]);
  const double r0 = v[0] + q[3] * t0 + (q[1] * t2 - q[2] * t1);
  const double r1 = v[1] + q[3] * t1 + (q[2] * t0 - q[0] * t2);
  const double r2 = v[2] + q[3] * t2 + (q[0] * t1 - q[1] * t0);
  out[0] = r0, out[1] = r1, out[2] = r2;
}

// quatMul (math.tsl.ts:17-23): a applied after b
__device__ __forceinline__ void quat_mul(const double a[4], const double b[4], double out[4]) {
  const double x = a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1];
  const double y = a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0];
  const double z = a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3];
  const double w = a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2];
  out[0] = x, out[1] = y, out[2] = z, out[3] = w;
}

// A zero quaternion normalises to the identity
__device__ __forceinline__ void quat_normalize(const double q[4], double out[4]) {
  const double l = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(l > 0.0)) {
    out[0] = out[1] = out[2] = 0.0;
    out[3] = 1.0;
    return;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) out[k] = q[k] / l;
}

// basisToQuat (math.tsl.ts:117-150): the w >= 0 quaternion of orthonormal columns x, y, z
__device__ void basis_to_quat(const double x[3], const double y[3], const double z[3], double q[4]) {
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
#pragma unroll
  for (int k = 0; k < 4; k++) q[k] /= l;
  if (q[3] < 0.0) {
#pragma unroll
    for (int k = 0; k < 4; k++) q[k] = -q[k];
  }
}

// scaleQuatMatrix (math.tsl.ts:25-44): column k is axis k of R(q) times s[k]
__device__ __forceinline__ void scale_quat_cols(const double s[3], const double q[4], double col[3][3]) {
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

// symEigens (src/gpu/math.tsl.ts:46-112): Jacobi rotations on the symmetric
// matrix (xx, yy, zz | xy, xz, yz), at most 16, stopping once every
// off-diagonal element is within 1e-6 of the diagonal's absolute sum;
// eigenvalues descending, eigenvectors (vec[i]) right-handed. A[c][r] and
// V[c][r] are column c, row r, as the reference indexes them.
__device__ void sym_eigens(const double d[3], const double o[3], double values[3], double vec[3][3]) {
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
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const double x = A[r][p], y = A[r][q];
      A[r][p] = c * x - sn * y;
      A[r][q] = sn * x + c * y;
    }
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const double x = A[p][r], y = A[q][r];
      A[p][r] = c * x - sn * y;
      A[q][r] = sn * x + c * y;
    }
    A[p][q] = 0.0;
    A[q][p] = 0.0;
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const double x = V[r][p], y = V[r][q];
      V[r][p] = c * x - sn * y;
      V[r][q] = sn * x + c * y;
    }
  }
  double l[3] = {A[0][0], A[1][1], A[2][2]};
  double v[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const double w[3] = {V[0][i], V[1][i], V[2][i]};
    const double len = sqrt(dot3(w, w));
#pragma unroll
    for (int k = 0; k < 3; k++) v[i][k] = w[k] / len;
  }
  const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int i = pairs[k][0], j = pairs[k][1];
    if (l[i] < l[j]) {
      const double t = l[i];
      l[i] = l[j];
      l[j] = t;
#pragma unroll
      for (int m = 0; m < 3; m++) {
        const double w = v[i][m];
        v[i][m] = v[j][m];
        v[j][m] = w;
      }
    }
  }
  const double cr[3] = {v[0][1] * v[1][2] - v[0][2] * v[1][1], v[0][2] * v[1][0] - v[0][0] * v[1][2],
                        v[0][0] * v[1][1] - v[0][1] * v[1][0]};
  if (dot3(cr, v[2]) < 0.0) {
#pragma unroll
    for (int k = 0; k < 3; k++) v[2][k] = -v[2][k];
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    values[k] = l[k];
#pragma unroll
    for (int m = 0; m < 3; m++) vec[k][m] = v[k][m];
  }
}

// P (column-major) times (c, 1), and times (v, 0)
__device__ __forceinline__ void clip_of(const double* P, const double c[3], double clip[4]) {
#pragma unroll
  for (int r = 0; r < 4; r++) clip[r] = P[r] * c[0] + P[4 + r] * c[1] + P[8 + r] * c[2] + P[12 + r];
}

__device__ __forceinline__ void proj_dir(const double* P, const double v[3], double out[4]) {
#pragma unroll
  for (int r = 0; r < 4; r++) out[r] = P[r] * v[0] + P[4 + r] * v[1] + P[8 + r] * v[2];
}

// The head-space splat form of an object-space covariance (row-major) seen
// through the object's 3x3 `a` (rows of 4): transformCov then fromCov
// (src/render/splatTransform.tsl.ts:117-140, src/gpu/splats.tsl.ts:189-199),
// the products in the oracle's order. Out of line: objects that take it are
// rare, and inlined its registers would weigh on every launch.
struct Cov3 {  // a symmetric 3x3, row-major
  double m[9];
};
struct SplatBasis {  // scales and rotation
  double s[3];
  double q[4];
};

__device__ __noinline__ SplatBasis cov_to_splat(const double* a, const Cov3 c) {
  const double* cov = c.m;
  double tmp[9], covh[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) tmp[i * 3 + j] = a[i * 4 + 0] * cov[0 * 3 + j] + a[i * 4 + 1] * cov[1 * 3 + j] + a[i * 4 + 2] * cov[2 * 3 + j];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) covh[i * 3 + j] = tmp[i * 3 + 0] * a[j * 4 + 0] + tmp[i * 3 + 1] * a[j * 4 + 1] + tmp[i * 3 + 2] * a[j * 4 + 2];
  const double d[3] = {covh[0], covh[4], covh[8]}, o[3] = {covh[3], covh[6], covh[7]};
  double values[3], v[3][3];
  sym_eigens(d, o, values, v);
  SplatBasis out;
#pragma unroll
  for (int k = 0; k < 3; k++) out.s[k] = sqrt(fmax(values[k], 0.0));
  basis_to_quat(v[0], v[1], v[2], out.q);
  return out;
}

struct Bound {  // projection.tsl.ts:206-210: ndc centre, angle, pixel half extents
  double ndc[2], angle, scales[2];
};

// eigenvector2 (projection.tsl.ts:215-219)
__device__ __forceinline__ void eigenvector2(double a, double b, double d, double eig, double v[2]) {
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

// boundFromCov (projection.tsl.ts:223-240)
__device__ bool bound_from_cov(double a, double b, double d, double std_dev, const DevParams& p, Bound& bd) {
  const double det = a * d - b * b;
  const double half = (a - d) * 0.5;
  const double eigen1 = (a + d) * 0.5 + sqrt(half * half + b * b);
  const double eigen2 = eigen1 > 0.0 ? fmax(det / eigen1, 0.0) : 0.0;
  const double scale1 = fmin((double)p.max_pixel_radius, std_dev * sqrt(fmax(eigen1, 0.0)));
  const double scale2 = fmin((double)p.max_pixel_radius, std_dev * sqrt(eigen2));
  const bool ok = scale1 >= (double)p.min_pixel_radius || scale2 >= (double)p.min_pixel_radius;
  if (ok) {
    double v[2];
    eigenvector2(a, b, d, eigen1, v);
    const double angle = atan2(v[1], v[0]);
    bd.angle = angle < 0.0 ? angle + 3.14159265358979323846 : angle;
    bd.scales[0] = scale1;
    bd.scales[1] = scale2;
  }
  return ok;
}

// screenBound (projection.tsl.ts:243-247)
__device__ __forceinline__ void screen_bound(const ProjDesc& sd, Bound& bd) {
  bd.ndc[0] = bd.ndc[1] = 0.0;
  bd.angle = 0.0;
  bd.scales[0] = bd.scales[1] =
      fmin((double)sd.params.max_pixel_radius, sqrt(sd.width * sd.width + sd.height * sd.height) * 0.5);
}

// clipBoundToScreen (projection.tsl.ts:250-273)
__device__ bool clip_bound_to_screen(const ProjDesc& sd, Bound& bd) {
  const double hx = sd.width * 0.5, hy = sd.height * 0.5;
  const double ca = cos(bd.angle), sa = sin(bd.angle);
  const double cx = ca * bd.scales[0], cy = ca * bd.scales[1], sx = sa * bd.scales[0], sy = sa * bd.scales[1];
  const double ex = sqrt(cx * cx + sy * sy), ey = sqrt(sx * sx + cy * cy);
  const double mx = bd.ndc[0] * hx, my = bd.ndc[1] * hy;
  double lox = mx - ex, loy = my - ey, hix = mx + ex, hiy = my + ey;
  if (!(lox >= -hx && loy >= -hy && hix <= hx && hiy <= hy)) {
    lox = fmax(lox, -hx);
    loy = fmax(loy, -hy);
    hix = fmin(hix, hx);
    hiy = fmin(hiy, hy);
    if (lox >= hix || loy >= hiy) return false;
    bd.ndc[0] = (lox + hix) * 0.5 / hx;
    bd.ndc[1] = (loy + hiy) * 0.5 / hy;
    bd.angle = 0.0;
    bd.scales[0] = (hix - lox) * 0.5;
    bd.scales[1] = (hiy - loy) * 0.5;
  }
  return true;
}

// ---- word codecs in float64 (projection.tsl.ts:277-366, src/gpu/encoding.tsl.ts) ----

__device__ __forceinline__ double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

__device__ __forceinline__ uint32_t fixed16(double v) {
  return (uint32_t)clampd(floor((v + 2.0) / 4.0 * 65535.0 + 0.5), 0.0, 65535.0);
}

// encodeLogScale (projection.tsl.ts:299-303) in `bits`, rounded up when outward
__device__ __forceinline__ uint32_t log_scale_code(double scale, int bits, bool outward) {
  const double top = (double)((1u << bits) - 2u);
  const double normalized = (clampd(log2(fmax(scale, 1e-20)), -4.0, 12.0) + 4.0) / 16.0 * top;
  return (uint32_t)clampd(outward ? ceil(normalized) : floor(normalized + 0.5), 0.0, top) + 1u;
}

// encodeBound (projection.tsl.ts:352-360): NDC 2x16; a 10-bit angle and two
// 11-bit log2 scales rounded outward, widened by the angle's half step
__device__ __forceinline__ void encode_bound(const Bound& bd, uint32_t w[2]) {
  const uint32_t angle_code = (uint32_t)floor(bd.angle / 3.14159265358979323846 * 1024.0 + 0.5) & 1023u;
  // sin(pi / 2048) * 1.001, the reference's constant in float64
  const double slack = fmax(bd.scales[0], bd.scales[1]) * (sin(3.14159265358979323846 / 1024.0 / 2.0) * 1.001);
  w[0] = fixed16(bd.ndc[0]) | (fixed16(bd.ndc[1]) << 16);
  w[1] = angle_code | (log_scale_code(bd.scales[0] + slack, 11, true) << 10) |
         (log_scale_code(bd.scales[1] + slack, 11, true) << 21);
}

// encodeCenter (projection.tsl.ts:317-332): the direction's top 16 + 16 bits,
// the float32 distance, and the low 4 + 4 bits at bits 24-31
__device__ __forceinline__ void encode_center(const double c[3], uint32_t w[3]) {
  const double distance = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
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
  w[0] = (qx >> 4) | ((qy >> 4) << 16);
  w[1] = __float_as_uint(__double2float_rn(distance));
  w[2] = ((qx & 15u) << 24) | (qy << 28);
}

// encodeOpacity (projection.tsl.ts:310): a nonzero byte
__device__ __forceinline__ uint32_t opacity_code(double opacity) {
  const uint32_t v = (uint32_t)floor(clampd(opacity * 128.0, 0.0, 255.0) + 0.5);
  return v > 1u ? v : 1u;
}

// Half bits of a float64, rounded to nearest even (Float16Array's rounding)
__device__ __forceinline__ uint32_t half_code(double f) { return (uint32_t)__half_as_ushort(__double2half(f)); }

// encodeExtRgb (encoding.tsl.ts:19-33): 8-bit magnitudes, 3 signs, a 5-bit shared exponent
__device__ uint32_t ext_rgb_code(const double rgb[3]) {
  const double max_abs = fmax(fabs(rgb[0]), fmax(fabs(rgb[1]), fabs(rgb[2])));
  int base = (max_abs > 0.0 ? (int)ceil(log2(max_abs)) : 0) + 15;
  base = base < 0 ? 0 : (base > 31 ? 31 : base);
  const double scale = 255.0 * ldexp(1.0, 15 - base);
  uint32_t m[3];
#pragma unroll
  for (int c = 0; c < 3; c++) m[c] = (uint32_t)fmin(floor(fabs(rgb[c]) * scale + 0.5), 255.0);
  const uint32_t signs = (rgb[0] < 0.0 ? 1u : 0u) | (rgb[1] < 0.0 ? 2u : 0u) | (rgb[2] < 0.0 ? 4u : 0u);
  return m[0] | (m[1] << 8) | (m[2] << 16) | ((((uint32_t)base << 3) | signs) << 24);
}

// encodeQuatOct32 (encoding.tsl.ts:69-117): a 10 + 10-bit octahedral axis of
// the w >= 0 quaternion, then its angle 0..pi in 12 bits
__device__ uint32_t quat_oct32_code(const double q[4]) {
  const double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(len > 0.0)) return 0u;
  const double s = (q[3] < 0.0 ? -1.0 : 1.0) / len;
  const double ax = q[0] * s, ay = q[1] * s, az = q[2] * s;
  const double angle = 2.0 * acos(fmin(1.0, q[3] * s));
  const uint32_t angle_code = (uint32_t)floor(angle / 3.14159265358979323846 * 4095.0 + 0.5);
  uint32_t axis = 0u;
  const double l1 = fabs(ax) + fabs(ay) + fabs(az);
  if (l1 > 0.0) {
    double px = ax / l1, py = ay / l1;
    if (az < 0.0) {
      const double fx = fabs(px);
      px = (1.0 - fabs(py)) * (px >= 0.0 ? 1.0 : -1.0);
      py = (1.0 - fx) * (py >= 0.0 ? 1.0 : -1.0);
    }
    axis = (uint32_t)floor((px * 0.5 + 0.5) * 1023.0 + 0.5) | ((uint32_t)floor((py * 0.5 + 0.5) * 1023.0 + 0.5) << 10);
    if (axis == 0u) axis = 0xfffffu;  // code 0 means "no vector": the same -Z
  }
  return axis | (angle_code << 20);
}

// ---- the bounds ----

// gutBound (projections.tsl.ts:183-220): the unscented transform of 7 sigma points
__device__ bool gut_bound(const ProjDesc& sd, const DevEye& e, const double ce[3], const double q[4], const double s[3],
                          double std_dev, Bound& bd) {
  const double r3 = sqrt(3.0);
  const double ss[3] = {s[0] * r3, s[1] * r3, s[2] * r3};
  double col[3][3];
  scale_quat_cols(ss, q, col);
  const double hx = sd.width * 0.5, hy = sd.height * 0.5;
  double px[7], py[7];
  bool in_front = true;
#pragma unroll
  for (int i = 0; i < 7; i++) {
    double pt[3] = {ce[0], ce[1], ce[2]};
    if (i > 0) {
      const double sign = (i & 1) ? 1.0 : -1.0;
#pragma unroll
      for (int k = 0; k < 3; k++) pt[k] = ce[k] + sign * col[(i - 1) / 2][k];
    }
    double clip[4];
    clip_of(e.proj, pt, clip);
    in_front = in_front && clip[3] > 0.0;
    px[i] = clip[0] / clip[3] * hx;
    py[i] = clip[1] / clip[3] * hy;
  }
  if (!in_front) {
    screen_bound(sd, bd);
    return true;
  }
  const double sixth = 1.0 / 6.0;
  double mx = 0.0, my = 0.0;
#pragma unroll
  for (int i = 1; i < 7; i++) {
    mx += px[i] * sixth;
    my += py[i] * sixth;
  }
  const double d0x = px[0] - mx, d0y = py[0] - my;
  double a = d0x * d0x * 2.0, b = d0x * d0y * 2.0, d = d0y * d0y * 2.0;
#pragma unroll
  for (int i = 1; i < 7; i++) {
    const double dx = px[i] - mx, dy = py[i] - my;
    a += dx * dx * sixth;
    b += dx * dy * sixth;
    d += dy * dy * sixth;
  }
  const bool ok = bound_from_cov(a, b, d, std_dev, sd.params, bd);
  bd.ndc[0] = mx / hx;
  bd.ndc[1] = my / hy;
  return ok;
}

// htgsBound (projections.tsl.ts:223-262): the exact outline of the std-dev ellipsoid
__device__ bool htgs_bound(const ProjDesc& sd, const DevEye& e, const double ce[3], const double ndc[2], const double q[4],
                           const double s[3], double std_dev, Bound& bd) {
  const double ss[3] = {s[0] * std_dev, s[1] * std_dev, s[2] * std_dev};
  double col[3][3], T[3][4], c3[4];
  scale_quat_cols(ss, q, col);
#pragma unroll
  for (int k = 0; k < 3; k++) proj_dir(e.proj, col[k], T[k]);
  clip_of(e.proj, ce, c3);
  const double xs[3] = {T[0][0], T[1][0], T[2][0]}, ys[3] = {T[0][1], T[1][1], T[2][1]},
               ws[3] = {T[0][3], T[1][3], T[2][3]};
  const double qww = dot3(ws, ws) - c3[3] * c3[3];
  bool valid = qww < 0.0 && c3[3] > 0.0;
  double cx = 0.0, cy = 0.0, a = 0.0, b = 0.0, d = 0.0;
  if (valid) {
    double u[3], v[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      u[k] = xs[k] * c3[3] - ws[k] * c3[0];
      v[k] = ys[k] * c3[3] - ws[k] * c3[1];
    }
    const double sww = dot3(ws, ws), xw = dot3(xs, ws), yw = dot3(ys, ws);
    const double inv_c2 = 1.0 / (qww * qww);
    const double hx = sd.width * 0.5, hy = sd.height * 0.5;
    a = (dot3(u, u) - (sww * dot3(xs, xs) - xw * xw)) * inv_c2 * hx * hx;
    b = (dot3(u, v) - (sww * dot3(xs, ys) - xw * yw)) * inv_c2 * hx * hy;
    d = (dot3(v, v) - (sww * dot3(ys, ys) - yw * yw)) * inv_c2 * hy * hy;
    cx = ndc[0] + dot3(ws, u) / (c3[3] * qww);
    cy = ndc[1] + dot3(ws, v) / (c3[3] * qww);
    valid = a > 0.0 && d > 0.0 && a * d - b * b > 0.0;
  }
  if (!valid) {
    screen_bound(sd, bd);
    return true;
  }
  const bool ok = bound_from_cov(a, b, d, 1.0, sd.params, bd);
  bd.ndc[0] = cx;
  bd.ndc[1] = cy;
  return ok;
}

// quadOffScreen (projections.tsl.ts:336-352)
__device__ bool quad_off_screen(const double* P, const double mu[3], const double a0[3], const double a1[3]) {
  double c[4], p0[4], p1[4];
  clip_of(P, mu, c);
  proj_dir(P, a0, p0);
  proj_dir(P, a1, p1);
  bool in_front = true, o0 = true, o1 = true, o2 = true, o3 = true;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double clip[4];
#pragma unroll
    for (int k = 0; k < 4; k++) clip[k] = c[k] + ((i & 1) ? p0[k] : -p0[k]) + ((i & 2) ? p1[k] : -p1[k]);
    in_front = in_front && clip[3] > 0.0;
    o0 = o0 && clip[0] < -clip[3];
    o1 = o1 && clip[0] > clip[3];
    o2 = o2 && clip[1] < -clip[3];
    o3 = o3 && clip[1] > clip[3];
  }
  return in_front && (o0 || o1 || o2 || o3);
}

// raygsFrame (projections.tsl.ts:356-397): the quad facing the eye
__device__ bool raygs_frame(const DevEye& e, const double ce[3], const double q[4], const double s[3], double std_dev,
                            double fq[4], double lengths[2], double& c2_out) {
  bool ok = true;
  const double kappa = std_dev * std_dev;
  const double conj[4] = {-q[0], -q[1], -q[2], q[3]};
  double local[3], mu[3];
  quat_rotate(conj, ce, local);
#pragma unroll
  for (int k = 0; k < 3; k++) local[k] /= s[k];
  double c2 = dot3(local, local);
  if (e.ortho) {
    const double back[3] = {0.0, 0.0, -1.0};
    double v[3];
    quat_rotate(conj, back, v);
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] /= s[k];
    const double l = sqrt(dot3(v, v));
#pragma unroll
    for (int k = 0; k < 3; k++) mu[k] = v[k] / l;
    c2 = 1e18;
  } else {
    ok = c2 > kappa * 1.0001;
    const double inv = 1.0 / sqrt(c2);
#pragma unroll
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
#pragma unroll
  for (int k = 0; k < 3; k++) {
    axis0[k] = q0[k] * u0[0] + q1[k] * u0[1];
    axis1[k] = q0[k] * u1[0] + q1[k] * u1[1];
  }
  lengths[0] = sqrt(dot3(axis0, axis0));
  lengths[1] = sqrt(dot3(axis1, axis1));
  ok = ok && lengths[0] > 0.0 && lengths[1] > 0.0;
  const double z_scale = std_dev / sqrt(fmax(1.0 - kappa / c2, 1e-4));
  double za0[3], za1[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    za0[k] = axis0[k] * z_scale;
    za1[k] = axis1[k] * z_scale;
  }
  ok = ok && !quad_off_screen(e.proj, ce, za0, za1);
  double n0[3], n1[3], n2[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    n0[k] = axis0[k] / lengths[0];
    n1[k] = axis1[k] / lengths[1];
  }
  n2[0] = n0[1] * n1[2] - n0[2] * n1[1];
  n2[1] = n0[2] * n1[0] - n0[0] * n1[2];
  n2[2] = n0[0] * n1[1] - n0[1] * n1[0];
  basis_to_quat(n0, n1, n2, fq);
  c2_out = c2;
  return ok;
}

// One splat: its words (row out_offset + i) and key. rayProjection.project /
// raygs.project (projections.tsl.ts:272-310, 405-432) behind
// SplatProjection.project / write (SplatProjection.ts:126-153).
template <int LAYOUT, int DEG, int VAR, int METHOD>
__device__ __forceinline__ void ray_one(const ProjDesc& sd, const RayDesc& rd, uint64_t i, uint32_t* __restrict__ words,
                                       uint32_t* __restrict__ keys) {
  const DevParams& p = sd.params;
  constexpr bool raygs = METHOD == kMethodRaygs;
  const int head_words = raygs ? 4 : 6, eye_words = raygs ? 3 : 2;
  const uint64_t gi = sd.out_offset + i;
  float cf[3], opac;
  double ls[3];
  bool zero_cov;
  load_head<LAYOUT>(sd.table, i, cf, opac, ls, zero_cov);
  double q[4];
  load_quat<LAYOUT>(sd.table, i, q);
  const double cx = cf[0], cy = cf[1], cz = cf[2];
  const double ch[3] = {affine_row(sd.a + 0, cx, cy, cz), affine_row(sd.a + 4, cx, cy, cz),
                        affine_row(sd.a + 8, cx, cy, cz)};
  double qn[4], qh[4], sc[3];
  quat_normalize(q, qn);
  if (LAYOUT != RDX_LAYOUT_COV && rd.uniform) {  // transformUniform (splatTransform.tsl.ts:143-152)
    quat_mul(rd.tq, qn, qh);
#pragma unroll
    for (int k = 0; k < 3; k++) sc[k] = exp(ls[k]) * rd.tscale;
  } else {
    // transformSplat's other branch (toCov, transformCov, fromCov), or a cov
    // table's transformCov and fromCov (transformForm / convertForm,
    // splatTransform.tsl.ts:154-181)
    Cov3 c3;
    double* cov = c3.m;
    if constexpr (LAYOUT == RDX_LAYOUT_COV) {
      double c6[6];
      load_cov(sd.table, i, c6);
      cov[0] = c6[0], cov[1] = c6[3], cov[2] = c6[4];
      cov[3] = c6[3], cov[4] = c6[1], cov[5] = c6[5];
      cov[6] = c6[4], cov[7] = c6[5], cov[8] = c6[2];
    } else {
      // covFromScaleQuat (math.tsl.ts:171-175): M M^T, M = R(q) diag(s)
      const double s0[3] = {exp(ls[0]), exp(ls[1]), exp(ls[2])};
      double col[3][3];
      scale_quat_cols(s0, qn, col);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) cov[r * 3 + c] = col[0][r] * col[0][c] + col[1][r] * col[1][c] + col[2][r] * col[2][c];
    }
    const SplatBasis b = cov_to_splat(sd.a, c3);
#pragma unroll
    for (int k = 0; k < 3; k++) sc[k] = b.s[k];
#pragma unroll
    for (int k = 0; k < 4; k++) qh[k] = b.q[k];
  }
  // prepareSplat, splat form (projection.tsl.ts:42-64), and cullInvisible (66-69)
  double opacity = opac, inflate = 1.0;
  if (opacity > 1.0) {
    opacity = fmin(opacity * 4.0 - 3.0, 5.0);
    if (p.lod_inflate) {
      inflate = pow(exp((opacity * opacity - 1.0) / 2.71828182845904523536), 1.0 / 3.0);
      opacity = 1.0;
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) sc[k] *= inflate;
  const double std_dev = opacity > 1.0 ? (double)p.max_std_dev + (opacity - 1.0) * 0.7 : (double)p.max_std_dev;
  const bool invisible =
      opacity <= 0.0 || opacity < (double)p.min_alpha || (sc[0] == 0.0 && sc[1] == 0.0 && sc[2] == 0.0);
  // the head: splatInView(headFrame()) with eye 0's lens (projection.tsl.ts:112-129)
  const DevEye& e0 = sd.eye[0];
  double hclip[4];
  clip_of(e0.proj, ch, hclip);
  double hblur = p.blur_amount;
  if (p.focal_distance > 0.0f && p.aperture_tan > 0.0f && ch[2] < 0.0) {
    const double depth = -ch[2];
    const double coc_view = fabs(depth - (double)p.focal_distance) * (double)p.aperture_tan;
    const double focal_pixels = sd.height * 0.5 * e0.proj[5];
    const double coc = e0.ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
    hblur = fmin(fmax(coc * coc, hblur), (double)p.max_pixel_radius * p.max_pixel_radius);
  }
  const double distance = sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
  bool guarded = true;
  if (p.sort_guard > 0.0f) {  // inSortGuard, splat form (projection.tsl.ts:145-155)
    const double radius = fmax(fmax(sc[0], sc[1]), sc[2]) * p.max_std_dev;
    const double w = fmax(hclip[3], 1e-6);
    const double rx = e0.proj[0] * radius / w, ry = e0.proj[5] * radius / w;
    const bool inside = fabs(hclip[0] / w) - rx <= (double)p.sort_guard + 1.0 &&
                        fabs(hclip[1] / w) - ry <= (double)p.sort_guard + 1.0;
    guarded = ch[2] < radius && (inside || -ch[2] <= radius);
  }
  // headBasis (projections.tsl.ts:173-180): viewBasis, then mipInflate (projection.tsl.ts:169-197)
  bool ok = !invisible;
  double op = opacity, hq[4], hs[3];
  quat_normalize(qh, hq);
  const double smax = fmax(sc[0], fmax(sc[1], sc[2])) * 1e-4;
#pragma unroll
  for (int k = 0; k < 3; k++) hs[k] = fmax(sc[k], smax);
  {
    const double conj[4] = {-hq[0], -hq[1], -hq[2], hq[3]};
    double local[3];
    quat_rotate(conj, ch, local);
    const double l2[3] = {local[0] * local[0], local[1] * local[1], local[2] * local[2]};
    const double pixel = 2.0 / (sd.height * e0.proj[5]);
    const double footprint = pixel * pixel * (e0.ortho ? 1.0 : dot3(ch, ch));
    double s2[3], s2b[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      s2[k] = hs[k] * hs[k] + (double)p.pre_blur_amount * footprint;
      s2b[k] = s2[k] + hblur * footprint;
    }
    const double num = l2[0] * s2[1] * s2[2] + l2[1] * s2[0] * s2[2] + l2[2] * s2[0] * s2[1];
    const double den = l2[0] * s2b[1] * s2b[2] + l2[1] * s2b[0] * s2b[2] + l2[2] * s2b[0] * s2b[1];
    op *= den > 0.0 ? sqrt(fmax(num / den, 0.0)) : 1.0;
#pragma unroll
    for (int k = 0; k < 3; k++) hs[k] = sqrt(s2b[k]);
  }
  ok = ok && op >= (double)p.min_alpha;
  uint32_t* row = words ? words + gi * (uint64_t)(head_words + sd.eyes * eye_words) : nullptr;
  bool any_visible = false;
  for (int v = 0; v < sd.eyes; v++) {
    const DevEye& e = sd.eye[v];
    uint32_t ew[3] = {0u, 0u, 0u};
    const double ce[3] = {affine_row(e.from_head + 0, ch[0], ch[1], ch[2]), affine_row(e.from_head + 4, ch[0], ch[1], ch[2]),
                          affine_row(e.from_head + 8, ch[0], ch[1], ch[2])};
    double clip[4];
    clip_of(e.proj, ce, clip);
    // cullDepth (projection.tsl.ts:132-134)
    const bool cull_depth = ce[2] >= 0.0 || clip[2] < sd.ndc_z_min * clip[3] || clip[2] >= clip[3];
    if (ok && !cull_depth) {
      double eq[4];
      quat_mul(rd.eye_q[v], hq, eq);  // frameQuat (projection.tsl.ts:101)
      if constexpr (raygs) {
        double fq[4], lengths[2], c2;
        if (raygs_frame(e, ce, eq, hs, std_dev, fq, lengths, c2)) {
          ew[0] = quat_oct32_code(fq);
          ew[1] = __float_as_uint(__double2float_rn(c2));
          ew[2] = half_code(log(lengths[0])) | (half_code(log(lengths[1])) << 16);
          any_visible = true;
        }
      } else {
        const double ndc[2] = {clip[3] > 0.0 ? clip[0] / clip[3] : 0.0, clip[3] > 0.0 ? clip[1] / clip[3] : 0.0};
        Bound bd = {{0.0, 0.0}, 0.0, {0.0, 0.0}};
        bool bound_ok;
        if constexpr (METHOD == kMethod3dgut) {
          bound_ok = gut_bound(sd, e, ce, eq, hs, std_dev, bd);
        } else {
          bound_ok = htgs_bound(sd, e, ce, ndc, eq, hs, std_dev, bd);
        }
        const bool on_screen = clip_bound_to_screen(sd, bd);
        if (bound_ok && on_screen) {
          encode_bound(bd, ew);
          any_visible = true;
        }
      }
    }
    if (row) {
      for (int k = 0; k < eye_words; k++) row[head_words + v * eye_words + k] = ew[k];
    }
  }
  if (row) {
    uint32_t hw[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    if (ok) {
      uint32_t c[3];
      encode_center(ch, c);
      const double stored = op > 1.0 ? (op + 3.0) * 0.25 : op;  // storedOpacity (projection.tsl.ts:72)
      // the base colour plus SH from the view origin (only the head words read it)
      double rgb[3];
      colour<LAYOUT, DEG, VAR>(sd.table, i, cx - sd.origin[0], cy - sd.origin[1], cz - sd.origin[2],
                               min(p.max_sh_degree, DEG), rgb);
      hw[0] = c[0];
      hw[1] = c[1];
      hw[2] = ext_rgb_code(rgb);
      if constexpr (raygs) {
        hw[3] = opacity_code(stored) | c[2];
      } else {
        hw[3] = quat_oct32_code(hq);
        hw[4] = half_code(log(hs[0])) | (half_code(log(hs[1])) << 16);
        hw[5] = half_code(log(hs[2])) | (opacity_code(stored) << 16) | c[2];
      }
    }
    for (int k = 0; k < head_words; k++) row[k] = hw[k];
  }
  // SplatProjection.write (SplatProjection.ts:150-151)
  const bool keyed = sd.cull_keys ? any_visible : (!invisible && guarded);
  if (keys) keys[gi] = keyed ? key_of_bits(__float_as_uint(__double2float_rn(distance)), sd.sort_bits) : invalid_key(sd.sort_bits);
}

// A warp per 32-splat tile of the launch's objects, grid-stride over the tiles
template <int LAYOUT, int DEG, int VAR, int METHOD>
__global__ void __launch_bounds__(kRayWarps * 32, 4) k_project_rays(const ProjDesc* __restrict__ descs,
                                                                  const RayDesc* __restrict__ rays, int n_desc,
                                                                  uint32_t total_tiles, uint32_t* __restrict__ words,
                                                                  uint32_t* __restrict__ keys) {
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * kRayWarps;
  for (uint32_t tile = blockIdx.x * kRayWarps + (threadIdx.x >> 5); tile < total_tiles; tile += stride) {
    int lo = 0, hi = n_desc - 1;  // the last descriptor whose first tile is at or before this one
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].first_tile <= tile) lo = mid;
      else hi = mid - 1;
    }
    const ProjDesc& sd = descs[lo];
    const uint64_t i = (uint64_t)(tile - sd.first_tile) * 32 + (uint64_t)lane;
    if (i < sd.count) ray_one<LAYOUT, DEG, VAR, METHOD>(sd, rays[lo], i, words, keys);
  }
}

using RayKernel = void (*)(const ProjDesc*, const RayDesc*, int, uint32_t, uint32_t*, uint32_t*);

template <int LAYOUT, int DEG, int VAR>
RayKernel ray_method(int method) {
  if (method == kMethod3dgut) return k_project_rays<LAYOUT, DEG, VAR, kMethod3dgut>;
  if (method == kMethodHtgs) return k_project_rays<LAYOUT, DEG, VAR, kMethodHtgs>;
  return k_project_rays<LAYOUT, DEG, VAR, kMethodRaygs>;
}

template <int LAYOUT, int VAR>
RayKernel ray_degree(int degree, int method) {
  switch (degree) {
    case 0: return ray_method<LAYOUT, 0, VAR>(method);
    case 1: return ray_method<LAYOUT, 1, VAR>(method);
    case 2: return ray_method<LAYOUT, 2, VAR>(method);
    case 3: return ray_method<LAYOUT, 3, VAR>(method);
    default: return ray_method<LAYOUT, 4, VAR>(method);
  }
}

template <int LAYOUT>
RayKernel ray_codec(int degree, int codec, int method) {
  if (codec == RDX_SH_PACKED && degree > 0) return ray_degree<LAYOUT, RDX_SH_PACKED>(degree, method);
  return ray_degree<LAYOUT, RDX_SH_EXT>(degree, method);
}

}  // namespace

cudaError_t launch_project_rays(const ProjDesc* descs_dev, const RayDesc* rays_dev, const ProjDesc* descs_host,
                                int n_desc, uint32_t total_tiles, int method, uint32_t* words, uint32_t* keys,
                                cudaStream_t stream) {
  if (total_tiles == 0 || n_desc == 0) return cudaSuccess;
  const DevTable& t = descs_host[0].table;  // one table kind per launch
  RayKernel k;
  switch (t.layout) {
    case RDX_LAYOUT_EXT: k = ray_codec<RDX_LAYOUT_EXT>(t.sh_degree, t.sh_codec, method); break;
    case RDX_LAYOUT_PACKED: k = ray_codec<RDX_LAYOUT_PACKED>(t.sh_degree, t.sh_codec, method); break;
    case RDX_LAYOUT_COV: k = ray_codec<RDX_LAYOUT_COV>(t.sh_degree, t.sh_codec, method); break;
    case RDX_LAYOUT_RAW:
      k = t.color_dtype == RDX_DTYPE_F16 ? ray_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F16>(t.sh_degree, method)
                                         : ray_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F32>(t.sh_degree, method);
      break;
    default: return cudaErrorInvalidValue;
  }
  const uint32_t grid = (total_tiles + kRayWarps - 1) / kRayWarps;
  k<<<grid, kRayWarps * 32, 0, stream>>>(descs_dev, rays_dev, n_desc, total_tiles, words, keys);
  return cudaGetLastError();
}

}  // namespace rdx
