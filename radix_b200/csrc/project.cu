// Fused per-splat projection for sm_100a: table decode, SH colour from the
// head (object space), object -> head transform, ewa projection per eye, the
// reference's words, float outputs, and the back-to-front sort key, one
// thread per splat in one launch over every object of a collection.
//
// Restates, fused: SplatProjector.build (src/render/SplatProjector.ts:153-194),
// SplatGenerator.fromSplats.withSh (src/gpu/splatGenerator.ts:152-158),
// GpuShReader.color/apply (src/gpu/sh.tsl.ts:255-266), transformCov
// (src/render/splatTransform.tsl.ts:120-140), prepareSplat / splatInView /
// culls (src/render/projection.tsl.ts:42-140), ewa.project
// (src/render/projections.tsl.ts:95-148) and SplatProjection.write
// (src/render/SplatProjection.ts:141-153).
//
// Precision: the head-space centre, the key distance and the centre culls
// (behind, near / far, clipXY) are float64 with explicitly rounded operations,
// so keys and cull decisions equal the float64 oracle's. Covariance, SH and
// bound maths are float32. The 2D covariance is factored as T T^T with
// T = J^T W R S (2 x 3): a = |t0|^2, d = |t1|^2, b = t0 . t1, and its
// determinant by Cauchy-Binet, sum over column pairs (j, k) of
// (s_j s_k m_l)^2 with m = u0 x u1 the cross product of the rows of J^T W R.
// Every term is non-negative, so thin splats keep float32 relative accuracy
// where a d - b^2 would cancel.
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

// Widest aligned vector that divides a row
template <int ROW_BYTES>
struct RowVec {
  static constexpr int bytes = ROW_BYTES % 16 == 0 ? 16 : (ROW_BYTES % 8 == 0 ? 8 : (ROW_BYTES % 4 == 0 ? 4 : 2));
};

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

// Base rgb + SH coefficients of one raw row as float32
template <int DEG, int CDT>
__device__ __forceinline__ void load_colors(const void* colors, uint64_t i, float* out) {
  constexpr int kValues = (1 + ShCount<DEG>::value) * 3;
  constexpr int kElem = CDT == RDX_DTYPE_F16 ? 2 : 4;
  constexpr int kRow = kValues * kElem;
  constexpr int kVec = RowVec<kRow>::bytes;
  alignas(16) unsigned char buf[(kRow + 15) / 16 * 16];
  const unsigned char* row = reinterpret_cast<const unsigned char*>(colors) + i * (uint64_t)kRow;
#pragma unroll
  for (int b = 0; b < kRow; b += kVec) load_vec<kVec>(row + b, buf + b);
#pragma unroll
  for (int v = 0; v < kValues; v++) {
    if constexpr (CDT == RDX_DTYPE_F16) {
      out[v] = __half2float(*reinterpret_cast<const __half*>(buf + v * 2));
    } else {
      out[v] = *reinterpret_cast<const float*>(buf + v * 4);
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

struct Splat {
  float3 center;
  float3 log_scales;
  float4 quat;
  float opacity;
  float3 rgb;
};

template <int LAYOUT, int DEG, int CDT, int EYES>
__global__ void __launch_bounds__(kProjThreads) k_project(const ProjDesc* __restrict__ descs, int n_desc,
                                                          ProjOutputs out) {
  __shared__ ProjDesc sd;
  __shared__ int s_desc;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int lo = 0, hi = n_desc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].first_tile <= blockIdx.x) {
        lo = mid;
      } else {
        hi = mid - 1;
      }
    }
    s_desc = lo;
  }
  __syncthreads();
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&descs[s_desc]);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sd);
    for (int w = tid; w < (int)(sizeof(ProjDesc) / 4); w += kProjThreads) dst[w] = src[w];
  }
  __syncthreads();
  const uint64_t i = (uint64_t)(blockIdx.x - sd.first_tile) * kProjThreads + tid;
  if (i >= sd.count) return;
  const DevTable& tb = sd.table;
  const DevParams& p = sd.params;
  constexpr int K = ShCount<DEG>::value;

  // ---- load one splat in object space ----
  // Colours stay exact until the float64 SH: raw values as float32 (f16 widens
  // exactly), ext colours as their words, decoded in float64 where used.
  Splat s;
  float sh[LAYOUT == RDX_LAYOUT_RAW && K > 0 ? K * 3 : 1];
  uint32_t shw[LAYOUT == RDX_LAYOUT_EXT && K > 0 ? K : 1];
  double base[3];
  if constexpr (LAYOUT == RDX_LAYOUT_EXT) {
    // src/core/splats.ts:10-24 layout; src/gpu/splats.tsl.ts:63-71 decode
    const uint4 A = __ldg(reinterpret_cast<const uint4*>(tb.ext_a) + i);
    const uint4 B = __ldg(reinterpret_cast<const uint4*>(tb.ext_b) + i);
    s.center = make_float3(__uint_as_float(A.x), __uint_as_float(A.y), __uint_as_float(A.z));
    s.opacity = (float)(A.w >> 24) * (1.0f / 128.0f);
    decode_ext_rgb_f64(B.x, base);
    s.log_scales = make_float3(half_bits_to_float(B.y), half_bits_to_float(B.y >> 16), half_bits_to_float(B.z));
    s.quat = decode_quat_oct32(B.w);
    if constexpr (K > 0) {
#pragma unroll
      for (int t = 0; t < (K + 3) / 4; t++) {
        const uint4 T = __ldg(reinterpret_cast<const uint4*>(tb.ext_sh[t]) + i);
        const uint32_t w4[4] = {T.x, T.y, T.z, T.w};
#pragma unroll
        for (int c = 0; c < 4; c++) {
          if (t * 4 + c < K) shw[t * 4 + c] = w4[c];
        }
      }
    }
  } else {
    const float* cp = tb.centers + i * 3;
    const float* lp = tb.log_scales + i * 3;
    s.center = make_float3(__ldg(cp), __ldg(cp + 1), __ldg(cp + 2));
    s.log_scales = make_float3(__ldg(lp), __ldg(lp + 1), __ldg(lp + 2));
    s.quat = __ldg(reinterpret_cast<const float4*>(tb.quats) + i);
    s.opacity = __ldg(tb.opacities + i);
    float col[(1 + K) * 3];
    load_colors<DEG, CDT>(tb.colors, i, col);
    base[0] = col[0];
    base[1] = col[1];
    base[2] = col[2];
#pragma unroll
    for (int v = 0; v < K * 3; v++) sh[v] = col[3 + v];
  }

  // ---- SH colour from the head, in object space, float64 ----
  // A table with SH gets rgb + SH clamped at 0 even when the cap draws no
  // band (GpuShReader.apply); without SH there is no reader and no clamp.
  if constexpr (K > 0) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int cap = min(p.max_sh_degree, DEG);
    if (cap >= 1) {
      const double dx = (double)s.center.x - sd.origin[0];
      const double dy = (double)s.center.y - sd.origin[1];
      const double dz = (double)s.center.z - sd.origin[2];
      const double l2 = dx * dx + dy * dy + dz * dz;
      const double inv = l2 > 0.0 ? 1.0 / sqrt(l2) : 0.0;
      const double x = dx * inv, y = dy * inv, z = dz * inv;
#pragma unroll
      for (int band = 1; band <= DEG; band++) {
        if (band <= cap) {
          double basis[9];
          const int nb = sh_basis_band(band, x, y, z, basis);
#pragma unroll
          for (int k = 0; k < 9; k++) {
            if (k < nb) {
              const int ci = band * band - 1 + k;
              double c[3];
              if constexpr (LAYOUT == RDX_LAYOUT_EXT) {
                decode_ext_rgb_f64(shw[ci], c);
              } else {
                c[0] = sh[ci * 3 + 0];
                c[1] = sh[ci * 3 + 1];
                c[2] = sh[ci * 3 + 2];
              }
              acc[0] = fma(c[0], basis[k], acc[0]);
              acc[1] = fma(c[1], basis[k], acc[1]);
              acc[2] = fma(c[2], basis[k], acc[2]);
            }
          }
        }
      }
    }
    s.rgb = make_float3((float)fmax(base[0] + acc[0], 0.0), (float)fmax(base[1] + acc[1], 0.0),
                        (float)fmax(base[2] + acc[2], 0.0));
  } else {
    s.rgb = make_float3((float)base[0], (float)base[1], (float)base[2]);
  }

  // ---- head-space centre and distance (float64) ----
  const double cx = s.center.x, cy = s.center.y, cz = s.center.z;
  const double hx = affine_row(sd.a + 0, cx, cy, cz);
  const double hy = affine_row(sd.a + 4, cx, cy, cz);
  const double hz = affine_row(sd.a + 8, cx, cy, cz);
  const double distance = __dsqrt_rn(dadd(dadd(dmul(hx, hx), dmul(hy, hy)), dmul(hz, hz)));

  // ---- prepareSplat: LoD stretch (projection.tsl.ts:42-64), float64 ----
  double opacity_d = s.opacity;
  double inflate2 = 1.0;  // inflate^2 multiplies the covariance
  if (opacity_d > 1.0) {
    opacity_d = fmin(opacity_d * 4.0 - 3.0, 5.0);
    if (p.lod_inflate) {
      inflate2 = exp((opacity_d * opacity_d - 1.0) * (2.0 / (3.0 * 2.718281828459045)));
      opacity_d = 1.0;
    }
  }
  const float opacity = (float)opacity_d;
  // scale^2 = exp(2 ln s), float64: the covariance needs more than float32
  // carries when its off-diagonal cancels
  const double s2x = exp(2.0 * (double)s.log_scales.x) * inflate2;
  const double s2y = exp(2.0 * (double)s.log_scales.y) * inflate2;
  const double s2z = exp(2.0 * (double)s.log_scales.z) * inflate2;
  const float std_dev = opacity_d > 1.0 ? (float)((double)p.max_std_dev + (opacity_d - 1.0) * 0.7) : p.max_std_dev;
  const bool degenerate = (s2x == 0.0 && s2y == 0.0 && s2z == 0.0) || sd.degenerate;
  const bool invisible = opacity_d <= 0.0 || opacity_d < (double)p.min_alpha || degenerate;

  // rotation R(q), row-major, float64 (src/gpu/math.tsl.ts:26-44 without the scales)
  double qx = s.quat.x, qy = s.quat.y, qz = s.quat.z, qw = s.quat.w;
  {
    const double ql2 = qx * qx + qy * qy + qz * qz + qw * qw;
    if (ql2 > 0.0) {
      const double inv = 1.0 / sqrt(ql2);
      qx *= inv;
      qy *= inv;
      qz *= inv;
      qw *= inv;
    } else {
      qx = qy = qz = 0.0;
      qw = 1.0;
    }
  }
  const double R[9] = {1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy - qw * qz), 2.0 * (qx * qz + qw * qy),
                       2.0 * (qx * qy + qw * qz), 1.0 - 2.0 * (qx * qx + qz * qz), 2.0 * (qy * qz - qw * qx),
                       2.0 * (qx * qz - qw * qy), 2.0 * (qy * qz + qw * qx), 1.0 - 2.0 * (qx * qx + qy * qy)};

  // ---- sort guard (only with params.sort_guard > 0; projection.tsl.ts:145-155) ----
  bool guarded = true;
  if (p.sort_guard > 0.0f) {
    // head-space covariance diagonal: |row_r(A3 R S)|^2
    const float sx = (float)sqrt(s2x), sy = (float)sqrt(s2y), sz = (float)sqrt(s2z);
    float ext2 = 0.0f;
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const float a0 = (float)sd.a[r * 4 + 0], a1 = (float)sd.a[r * 4 + 1], a2 = (float)sd.a[r * 4 + 2];
      const float g0 = (a0 * (float)R[0] + a1 * (float)R[3] + a2 * (float)R[6]) * sx;
      const float g1 = (a0 * (float)R[1] + a1 * (float)R[4] + a2 * (float)R[7]) * sy;
      const float g2 = (a0 * (float)R[2] + a1 * (float)R[5] + a2 * (float)R[8]) * sz;
      ext2 = fmaxf(ext2, g0 * g0 + g1 * g1 + g2 * g2);
    }
    const float radius = sqrtf(ext2) * p.max_std_dev;
    const double* P = sd.eye[0].proj;
    const float clx = (float)(P[0] * hx + P[4] * hy + P[8] * hz + P[12]);
    const float cly = (float)(P[1] * hx + P[5] * hy + P[9] * hz + P[13]);
    const float clw = (float)(P[3] * hx + P[7] * hy + P[11] * hz + P[15]);
    const float w = fmaxf(clw, 1e-6f);
    const float rx = (float)P[0] * radius / w, ry = (float)P[5] * radius / w;
    const bool inside = fabsf(clx / w) - rx <= p.sort_guard + 1.0f && fabsf(cly / w) - ry <= p.sort_guard + 1.0f;
    const bool near_head = -(float)hz <= radius;
    guarded = (float)hz < radius && (inside || near_head);
  }

  const uint64_t gi = sd.out_offset + i;
  bool any_visible = false;
  if (!sd.keys_only) {
#pragma unroll
    for (int v = 0; v < EYES; v++) {
      const DevEye& e = sd.eye[v];
      // splatInView (projection.tsl.ts:112-129), float64 centre and clip
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
      const double limit = dmul(fmin((double)p.clip_xy, 2.0), clw);
      bool ok = !(invisible || ez >= 0.0 || clz < dmul(sd.ndc_z_min, clw) || clz >= clw || fabs(clx) > limit ||
                  fabs(cly) > limit);
      const float fz = (float)ez;
      float blur = p.blur_amount;
      if (p.focal_distance > 0.0f && p.aperture_tan > 0.0f && fz < 0.0f) {
        const float depth = -fz;
        const float coc_view = fabsf(depth - p.focal_distance) * p.aperture_tan;
        const float focal_pixels = (float)sd.height * 0.5f * e.proj11;
        const float coc = e.ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
        blur = fminf(fmaxf(coc * coc, blur), p.max_pixel_radius * p.max_pixel_radius);
      }
      double ndcx_d = 0.0, ndcy_d = 0.0;
      if (clw > 0.0) {
        const double inv_w = 1.0 / clw;
        ndcx_d = clx * inv_w;
        ndcy_d = cly * inv_w;
      }
      const float ndcx = (float)ndcx_d, ndcy = (float)ndcy_d;
      float a = 0.f, b = 0.f, d = 0.f, det = 0.f, opacity_c = 0.f, scale1 = 0.f, scale2 = 0.f, angle = 0.f;
      double a_d = 0.0, b_d = 0.0, d_d = 0.0, det_d = 1.0;
      if (ok) {
        // J (projections.tsl.ts:108-118), float64
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
        // rows of J^T W (W = object -> eye 3x3), then of J^T W R
        const double* W = e.wd;
        const double w0x = j1x * W[0] + j2x * W[6], w0y = j1x * W[1] + j2x * W[7], w0z = j1x * W[2] + j2x * W[8];
        const double w1x = j1y * W[3] + j2y * W[6], w1y = j1y * W[4] + j2y * W[7], w1z = j1y * W[5] + j2y * W[8];
        const double u00 = w0x * R[0] + w0y * R[3] + w0z * R[6];
        const double u01 = w0x * R[1] + w0y * R[4] + w0z * R[7];
        const double u02 = w0x * R[2] + w0y * R[5] + w0z * R[8];
        const double u10 = w1x * R[0] + w1y * R[3] + w1z * R[6];
        const double u11 = w1x * R[1] + w1y * R[4] + w1z * R[7];
        const double u12 = w1x * R[2] + w1y * R[5] + w1z * R[8];
        // cov2D = T T^T with T = U S: a = sum u0k^2 s_k^2, d = sum u1k^2 s_k^2, b = sum u0k u1k s_k^2
        const double ra = u00 * u00 * s2x + u01 * u01 * s2y + u02 * u02 * s2z;
        const double rd = u10 * u10 * s2x + u11 * u11 * s2y + u12 * u12 * s2z;
        const double rb = u00 * u10 * s2x + u01 * u11 * s2y + u02 * u12 * s2z;
        // det(T T^T) by Cauchy-Binet: sum over column pairs of (s_j s_k (u0 x u1)_l)^2
        const double m0 = u01 * u12 - u02 * u11;
        const double m1 = u02 * u10 - u00 * u12;
        const double m2 = u00 * u11 - u01 * u10;
        const double det_t = m0 * m0 * (s2y * s2z) + m1 * m1 * (s2x * s2z) + m2 * m2 * (s2x * s2y);
        const double pre = p.pre_blur_amount, full = (double)p.pre_blur_amount + (double)blur;
        const double det_orig = det_t + pre * (ra + rd) + pre * pre;
        det_d = det_t + full * (ra + rd) + full * full;
        a_d = ra + full;
        d_d = rd + full;
        b_d = rb;
        const double opacity_cd = opacity_d * sqrt(fmax(0.0, det_orig / det_d));
        opacity_c = (float)opacity_cd;
        const double contribution = opacity_cd * 6.283185307179586 * sqrt(fmax(0.0, det_d));
        a = (float)a_d;
        b = (float)b_d;
        d = (float)d_d;
        det = (float)det_d;
        // boundFromCov (projection.tsl.ts:223-240)
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
      const uint64_t ei = (uint64_t)v * sd.out_n + gi;
      if (ok) {
        const double inv_det = 1.0 / det_d;
        if (out.mean2d) {
          reinterpret_cast<float2*>(out.mean2d)[ei] =
              make_float2((float)((ndcx_d + 1.0) * 0.5 * sd.width), (float)((ndcy_d + 1.0) * 0.5 * sd.height));
        }
        if (out.conic) {
          out.conic[ei * 3 + 0] = (float)(d_d * inv_det);
          out.conic[ei * 3 + 1] = (float)(-b_d * inv_det);
          out.conic[ei * 3 + 2] = (float)(a_d * inv_det);
        }
        if (out.depth) out.depth[ei] = -fz;
        if (out.opacity) out.opacity[ei] = opacity_c;
        if (out.rgb) {
          out.rgb[ei * 3 + 0] = s.rgb.x;
          out.rgb[ei * 3 + 1] = s.rgb.y;
          out.rgb[ei * 3 + 2] = s.rgb.z;
        }
        if (out.radii) {
          out.radii[ei * 3 + 0] = scale1;
          out.radii[ei * 3 + 1] = scale2;
          out.radii[ei * 3 + 2] = angle;
        }
        if (out.words) {
          const float stored = opacity_c > 1.0f ? (opacity_c + 3.0f) * 0.25f : opacity_c;
          uint4 wv;
          wv.x = encode_fixed16(ndcx) | (encode_fixed16(ndcy) << 16);
          wv.y = encode_depth20(fz) | (encode_angle12(angle) << 20);
          wv.z = encode_ext_rgb(s.rgb.x, s.rgb.y, s.rgb.z);
          wv.w = encode_opacity8(stored) | (encode_log_scale12(scale1) << 8) | (encode_log_scale12(scale2) << 20);
          reinterpret_cast<uint4*>(out.words)[gi * EYES + v] = wv;
        }
        any_visible = true;
      } else {
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
  if (out.keys) {
    const bool keyed = sd.cull_keys && !sd.keys_only ? any_visible : (!invisible && guarded);
    out.keys[gi] = keyed ? key_of_bits(__float_as_uint(__double2float_rn(distance)), sd.sort_bits)
                         : invalid_key(sd.sort_bits);
  }
}

using ProjKernel = void (*)(const ProjDesc*, int, ProjOutputs);

template <int LAYOUT, int DEG, int CDT>
ProjKernel pick_eyes(int eyes) {
  return eyes == 2 ? k_project<LAYOUT, DEG, CDT, 2> : k_project<LAYOUT, DEG, CDT, 1>;
}

template <int LAYOUT, int CDT>
ProjKernel pick_degree(int degree, int eyes) {
  switch (degree) {
    case 0: return pick_eyes<LAYOUT, 0, CDT>(eyes);
    case 1: return pick_eyes<LAYOUT, 1, CDT>(eyes);
    case 2: return pick_eyes<LAYOUT, 2, CDT>(eyes);
    case 3: return pick_eyes<LAYOUT, 3, CDT>(eyes);
    default: return pick_eyes<LAYOUT, 4, CDT>(eyes);
  }
}

ProjKernel pick_kernel(int layout, int degree, int cdt, int eyes) {
  if (layout == RDX_LAYOUT_EXT) return pick_degree<RDX_LAYOUT_EXT, RDX_DTYPE_F32>(degree, eyes);
  if (cdt == RDX_DTYPE_F16) return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F16>(degree, eyes);
  return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F32>(degree, eyes);
}

}  // namespace

cudaError_t launch_project(const ProjDesc* descs_dev, const ProjDesc* descs_host, int n_desc, uint32_t total_tiles,
                           const ProjOutputs& out, cudaStream_t stream) {
  if (total_tiles == 0 || n_desc == 0) return cudaSuccess;
  // One kernel per launch: the caller groups objects by table kind
  const ProjDesc& d0 = descs_host[0];
  ProjKernel k = pick_kernel(d0.table.layout, d0.table.sh_degree, d0.table.color_dtype, d0.eyes);
  k<<<total_tiles, kProjThreads, 0, stream>>>(descs_dev, n_desc, out);
  return cudaGetLastError();
}

}  // namespace rdx
