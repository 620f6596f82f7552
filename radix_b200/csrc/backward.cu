// Gradient of the fused projection for sm_100a: for raw float32 tables, the
// adjoint of mean2d, conic, depth, opacity and rgb (per eye) with respect to
// each splat's centre, ln scales, stored quaternion, opacity and colour rows
// (base rgb and SH coefficients). No counterpart in the reference, which only
// renders; it differentiates the path restated from projection.tsl.ts:42-140,
// projections.tsl.ts:95-148, sh.tsl.ts:60-139 and splatGenerator.ts:152-158.
//
// One thread per splat, float64 throughout: the forward values the adjoint
// needs are recomputed from the table (centre transform, J, the covariance
// factor T = J^T W R S, the blurred 2D covariance), then propagated back
// through T to R, S and J, through J to the eye-space centre, and through
// the SH basis and the normalised direction to the centre again. An eye
// whose forward opacity output is 0 did not draw the splat and contributes
// nothing; the rgb clamp passes a gradient only where base + SH > 0.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr int kBwdThreads = 128;
constexpr int kBwdBlocksPerSm = 4;  // 128 registers a thread (some spills: faster than 3 blocks of 168)

template <int DEG>
struct Coeffs {
  static constexpr int value = DEG == 0 ? 0 : (DEG == 1 ? 3 : (DEG == 2 ? 8 : (DEG == 3 ? 15 : 24)));
};

// The 3DGS basis (src/gpu/sh.tsl.ts:60-102) and its derivative with respect
// to (x, y, z) as polynomials, for the first K functions
template <int K>
__device__ __forceinline__ void sh_basis_and_grad(double x, double y, double z, double* Y, double (*G)[3]) {
  const double xx = x * x, yy = y * y, zz = z * z;
  const double c1 = 0.4886025, c2a = 1.0925484, c2b = 0.3153916, c2c = 0.5462742;
  const double c3a = 0.5900436, c3b = 2.8906114, c3c = 0.4570458, c3d = 0.3731763, c3e = 1.4453057;
  const double c4a = 2.5033429, c4b = 1.7701308, c4c = 0.9461747, c4d = 0.6690465, c4e = 0.1057855,
               c4f = 0.4730873, c4g = 0.6258357;
  auto set = [&](int k, double y_, double gx, double gy, double gz) {
    Y[k] = y_;
    G[k][0] = gx;
    G[k][1] = gy;
    G[k][2] = gz;
  };
  if (K > 0) {
    set(0, -c1 * y, 0.0, -c1, 0.0);
    set(1, c1 * z, 0.0, 0.0, c1);
    set(2, -c1 * x, -c1, 0.0, 0.0);
  }
  if (K > 3) {
    set(3, c2a * x * y, c2a * y, c2a * x, 0.0);
    set(4, -c2a * y * z, 0.0, -c2a * z, -c2a * y);
    set(5, c2b * (2.0 * zz - xx - yy), -2.0 * c2b * x, -2.0 * c2b * y, 4.0 * c2b * z);
    set(6, -c2a * x * z, -c2a * z, 0.0, -c2a * x);
    set(7, c2c * (xx - yy), 2.0 * c2c * x, -2.0 * c2c * y, 0.0);
  }
  if (K > 8) {
    set(8, -c3a * y * (3.0 * xx - yy), -6.0 * c3a * x * y, -3.0 * c3a * (xx - yy), 0.0);
    set(9, c3b * x * y * z, c3b * y * z, c3b * x * z, c3b * x * y);
    set(10, -c3c * y * (4.0 * zz - xx - yy), 2.0 * c3c * x * y, -c3c * (4.0 * zz - xx - 3.0 * yy), -8.0 * c3c * y * z);
    set(11, c3d * z * (2.0 * zz - 3.0 * xx - 3.0 * yy), -6.0 * c3d * x * z, -6.0 * c3d * y * z,
        c3d * (6.0 * zz - 3.0 * xx - 3.0 * yy));
    set(12, -c3c * x * (4.0 * zz - xx - yy), -c3c * (4.0 * zz - 3.0 * xx - yy), 2.0 * c3c * x * y, -8.0 * c3c * x * z);
    set(13, c3e * z * (xx - yy), 2.0 * c3e * x * z, -2.0 * c3e * y * z, c3e * (xx - yy));
    set(14, -c3a * x * (xx - 3.0 * yy), -3.0 * c3a * (xx - yy), 6.0 * c3a * x * y, 0.0);
  }
  if (K > 15) {
    const double zz7m1 = 7.0 * zz - 1.0, zz7m3 = 7.0 * zz - 3.0;
    set(15, c4a * x * y * (xx - yy), c4a * (3.0 * xx * y - yy * y), c4a * (xx * x - 3.0 * x * yy), 0.0);
    set(16, -c4b * y * z * (3.0 * xx - yy), -6.0 * c4b * x * y * z, -3.0 * c4b * z * (xx - yy),
        -c4b * y * (3.0 * xx - yy));
    set(17, c4c * x * y * zz7m1, c4c * y * zz7m1, c4c * x * zz7m1, 14.0 * c4c * x * y * z);
    set(18, -c4d * y * z * zz7m3, 0.0, -c4d * z * zz7m3, -c4d * y * (21.0 * zz - 3.0));
    set(19, c4e * (zz * (35.0 * zz - 30.0) + 3.0), 0.0, 0.0, c4e * (140.0 * zz * z - 60.0 * z));
    set(20, -c4d * x * z * zz7m3, -c4d * z * zz7m3, 0.0, -c4d * x * (21.0 * zz - 3.0));
    set(21, c4f * (xx - yy) * zz7m1, 2.0 * c4f * x * zz7m1, -2.0 * c4f * y * zz7m1, 14.0 * c4f * z * (xx - yy));
    set(22, -c4b * x * z * (xx - 3.0 * yy), -3.0 * c4b * z * (xx - yy), 6.0 * c4b * x * y * z,
        -c4b * x * (xx - 3.0 * yy));
    set(23, c4g * (xx * (xx - 3.0 * yy) - yy * (3.0 * xx - yy)), c4g * (4.0 * xx * x - 12.0 * x * yy),
        c4g * (4.0 * yy * y - 12.0 * xx * y), 0.0);
  }
}

template <int DEG, int CDT>
__device__ __forceinline__ double colour_value(const void* colors, uint64_t i, int j) {
  constexpr int kRow = (1 + Coeffs<DEG>::value) * 3;
  if constexpr (CDT == RDX_DTYPE_F16) {
    return (double)__half2float(reinterpret_cast<const __half*>(colors)[i * kRow + j]);
  } else {
    return (double)__ldg(reinterpret_cast<const float*>(colors) + i * kRow + j);
  }
}

// The gradient of row i of an object (drawn: the eyes whose forward drew it,
// not 0). col: the row's colour values (base rgb, then the SH coefficients),
// staged in shared memory; the row's colour gradient replaces them there.
template <int DEG, int CDT, int EYES>
__device__ __forceinline__ void splat_backward(const ProjDesc& sd, const GradsOut& go_, const GradsIn& in, uint64_t i,
                                               uint32_t drawn, float* col) {
  constexpr int K = Coeffs<DEG>::value;
  const uint64_t gi = sd.out_offset + i;
  const DevParams& p = sd.params;
  const DevTable& tb = sd.table;

  double g_c[3] = {0.0, 0.0, 0.0}, g_S[3] = {0.0, 0.0, 0.0}, g_R[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double g_op = 0.0, g_rgb[3] = {0.0, 0.0, 0.0};
  // the splat
  const double cx = __ldg(tb.centers + i * 3), cy = __ldg(tb.centers + i * 3 + 1), cz = __ldg(tb.centers + i * 3 + 2);
  const double ls0 = __ldg(tb.log_scales + i * 3), ls1 = __ldg(tb.log_scales + i * 3 + 1),
               ls2 = __ldg(tb.log_scales + i * 3 + 2);
  const double opac = __ldg(tb.opacities + i);
  double qn[4];
  const float4 q4 = __ldg(reinterpret_cast<const float4*>(tb.quats) + i);
  qn[0] = q4.x;
  qn[1] = q4.y;
  qn[2] = q4.z;
  qn[3] = q4.w;
  const double ql = sqrt(qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]);
  const bool qvalid = ql > 0.0;
  if (qvalid) {
    const double qi = 1.0 / ql;
#pragma unroll
    for (int k = 0; k < 4; k++) qn[k] *= qi;
  } else {
    qn[0] = qn[1] = qn[2] = 0.0;
    qn[3] = 1.0;
  }
  const double qx = qn[0], qy = qn[1], qz = qn[2], qw = qn[3];
  const double R[9] = {1.0 - 2.0 * (qy * qy + qz * qz), 2.0 * (qx * qy - qw * qz), 2.0 * (qx * qz + qw * qy),
                       2.0 * (qx * qy + qw * qz), 1.0 - 2.0 * (qx * qx + qz * qz), 2.0 * (qy * qz - qw * qx),
                       2.0 * (qx * qz - qw * qy), 2.0 * (qy * qz + qw * qx), 1.0 - 2.0 * (qx * qx + qy * qy)};
  // prepareSplat (projection.tsl.ts:42-64): the LoD stretch and inflation
  double op = opac, infl2 = 1.0, dop_do = 1.0;
  bool op_const = false;
  if (op > 1.0) {
    const double raw = op * 4.0 - 3.0;
    dop_do = raw < 5.0 ? 4.0 : 0.0;
    op = fmin(raw, 5.0);
    if (p.lod_inflate) {
      infl2 = exp((op * op - 1.0) * (2.0 / (3.0 * 2.718281828459045)));
      op_const = true;
    }
  }
  const double op_used = op_const ? 1.0 : op;
  const double sinfl = sqrt(infl2);
  const double S[3] = {exp(ls0) * sinfl, exp(ls1) * sinfl, exp(ls2) * sinfl};
  const double hx = affine_row(sd.a + 0, cx, cy, cz);
  const double hy = affine_row(sd.a + 4, cx, cy, cz);
  const double hz = affine_row(sd.a + 8, cx, cy, cz);

  {
#pragma unroll
    for (int v = 0; v < EYES; v++) {
      if (!((drawn >> v) & 1u)) continue;
      const DevEye& e = sd.eye[v];
      const uint64_t ei = (uint64_t)v * sd.out_n + gi;
      double ex = hx, ey = hy, ez = hz;
      if (!e.identity) {
        ex = affine_row(e.from_head + 0, hx, hy, hz);
        ey = affine_row(e.from_head + 4, hx, hy, hz);
        ez = affine_row(e.from_head + 8, hx, hy, hz);
      }
      const double* P = e.proj;
      const double clx = P[0] * ex + P[4] * ey + P[8] * ez + P[12];
      const double cly = P[1] * ex + P[5] * ey + P[9] * ez + P[13];
      const double clw = P[3] * ex + P[7] * ey + P[11] * ez + P[15];
      const double ndcx = clx / clw, ndcy = cly / clw;
      // the depth-of-field blur (projection.tsl.ts:117-125) and its derivative in the depth
      double blur = p.blur_amount, dblur = 0.0;
      if (p.focal_distance > 0.0f && p.aperture_tan > 0.0f && ez < 0.0) {
        const double depth = -ez;
        const double dist = depth - (double)p.focal_distance;
        const double focal_pixels = sd.height * 0.5 * e.proj[5];
        const double coc_view = fabs(dist) * (double)p.aperture_tan;
        const double coc = e.ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
        const double maxr2 = (double)p.max_pixel_radius * p.max_pixel_radius;
        const double c2 = coc * coc;
        if (c2 > blur && c2 < maxr2) {
          const double sgn = dist >= 0.0 ? 1.0 : -1.0;
          const double dcoc = e.ortho ? sgn * p.aperture_tan * focal_pixels
                                      : sgn * p.aperture_tan * focal_pixels / depth - coc / depth;
          dblur = 2.0 * coc * dcoc;
        }
        blur = fmin(fmax(c2, blur), maxr2);
      }
      // J, M = J^T W rows, U = M R, T = U S (the forward's factor of the 2D covariance)
      const double fx = e.focal_d[0], fy = e.focal_d[1];
      double j1x, j1y, j2x = 0.0, j2y = 0.0;
      if (e.ortho) {
        j1x = fx;
        j1y = fy;
      } else {
        const double inv_z = 1.0 / ez;
        j1x = fx * inv_z;
        j1y = fy * inv_z;
        j2x = -(j1x * ex) * inv_z;
        j2y = -(j1y * ey) * inv_z;
      }
      const double* Wm = e.wd;
      const double w0[3] = {j1x * Wm[0] + j2x * Wm[6], j1x * Wm[1] + j2x * Wm[7], j1x * Wm[2] + j2x * Wm[8]};
      const double w1[3] = {j1y * Wm[3] + j2y * Wm[6], j1y * Wm[4] + j2y * Wm[7], j1y * Wm[5] + j2y * Wm[8]};
      double U0[3], U1[3], T0[3], T1[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        U0[k] = w0[0] * R[k] + w0[1] * R[3 + k] + w0[2] * R[6 + k];
        U1[k] = w1[0] * R[k] + w1[1] * R[3 + k] + w1[2] * R[6 + k];
        T0[k] = U0[k] * S[k];
        T1[k] = U1[k] * S[k];
      }
      const double ra = T0[0] * T0[0] + T0[1] * T0[1] + T0[2] * T0[2];
      const double rd = T1[0] * T1[0] + T1[1] * T1[1] + T1[2] * T1[2];
      const double b = T0[0] * T1[0] + T0[1] * T1[1] + T0[2] * T1[2];
      const double pre = p.pre_blur_amount, full = (double)p.pre_blur_amount + blur;
      const double a = ra + full, d = rd + full;
      const double det = a * d - b * b;
      const double det_orig = (ra + pre) * (rd + pre) - b * b;
      const double r = det_orig / det;

      // ---- adjoint of this eye's outputs ----
      const double gm0 = in.mean2d ? (double)__ldg(in.mean2d + ei * 2) : 0.0;
      const double gm1 = in.mean2d ? (double)__ldg(in.mean2d + ei * 2 + 1) : 0.0;
      const double gc0 = in.conic ? (double)__ldg(in.conic + ei * 3) : 0.0;
      const double gc1 = in.conic ? (double)__ldg(in.conic + ei * 3 + 1) : 0.0;
      const double gc2 = in.conic ? (double)__ldg(in.conic + ei * 3 + 2) : 0.0;
      const double gd = in.depth ? (double)__ldg(in.depth + ei) : 0.0;
      const double go = in.opacity ? (double)__ldg(in.opacity + ei) : 0.0;
      if (in.rgb) {
#pragma unroll
        for (int c = 0; c < 3; c++) g_rgb[c] += (double)__ldg(in.rgb + ei * 3 + c);
      }
      // conic = (d, -b, a) / det; opacity = op sqrt(det_orig / det)
      double G_a = gc2 / det, G_d = gc0 / det, G_b = -gc1 / det;
      double G_det = (-gc0 * d + gc1 * b - gc2 * a) / (det * det);
      double G_do = 0.0;
      if (r > 0.0) {
        const double sr = sqrt(r);
        g_op += go * sr;
        const double G_r = go * op_used / (2.0 * sr);
        G_do = G_r / det;
        G_det -= G_r * r / det;
      }
      G_a += G_det * d;
      G_d += G_det * a;
      G_b -= 2.0 * b * G_det;
      const double G_ra = G_a + G_do * (rd + pre), G_rd = G_d + G_do * (ra + pre);
      G_b -= 2.0 * b * G_do;
      const double G_blur = G_a + G_d;
      // ra, rd, b from T; T = U S; U = M R
      double gw0[3] = {0.0, 0.0, 0.0}, gw1[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double gT0 = 2.0 * G_ra * T0[k] + G_b * T1[k];
        const double gT1 = 2.0 * G_rd * T1[k] + G_b * T0[k];
        g_S[k] += gT0 * U0[k] + gT1 * U1[k];
        const double gU0 = gT0 * S[k], gU1 = gT1 * S[k];
#pragma unroll
        for (int j = 0; j < 3; j++) {
          g_R[j * 3 + k] += w0[j] * gU0 + w1[j] * gU1;
          gw0[j] += gU0 * R[j * 3 + k];
          gw1[j] += gU1 * R[j * 3 + k];
        }
      }
      // M rows from J: w0 = j1x W0 + j2x W2, w1 = j1y W1 + j2y W2
      const double g_j1x = gw0[0] * Wm[0] + gw0[1] * Wm[1] + gw0[2] * Wm[2];
      const double g_j2x = gw0[0] * Wm[6] + gw0[1] * Wm[7] + gw0[2] * Wm[8];
      const double g_j1y = gw1[0] * Wm[3] + gw1[1] * Wm[4] + gw1[2] * Wm[5];
      const double g_j2y = gw1[0] * Wm[6] + gw1[1] * Wm[7] + gw1[2] * Wm[8];
      double g_e[3] = {0.0, 0.0, 0.0};
      if (!e.ortho) {
        const double z2 = ez * ez, z3 = z2 * ez;
        g_e[0] += g_j2x * (-fx / z2);
        g_e[1] += g_j2y * (-fy / z2);
        g_e[2] += g_j1x * (-fx / z2) + g_j1y * (-fy / z2) + g_j2x * (2.0 * fx * ex / z3) + g_j2y * (2.0 * fy * ey / z3);
      }
      g_e[2] -= G_blur * dblur;  // depth = -z
      // mean2d = (ndc + 1) / 2 * size, ndc = clip.xy / clip.w; depth = -z
      const double gn0 = gm0 * 0.5 * sd.width, gn1 = gm1 * 0.5 * sd.height;
      const double gcx = gn0 / clw, gcy = gn1 / clw, gcw = -(gn0 * ndcx + gn1 * ndcy) / clw;
      g_e[0] += P[0] * gcx + P[1] * gcy + P[3] * gcw;
      g_e[1] += P[4] * gcx + P[5] * gcy + P[7] * gcw;
      g_e[2] += P[8] * gcx + P[9] * gcy + P[11] * gcw - gd;
      // e = W c + const (W = fromHead_3 A_3)
#pragma unroll
      for (int c = 0; c < 3; c++) g_c[c] += Wm[c] * g_e[0] + Wm[3 + c] * g_e[1] + Wm[6 + c] * g_e[2];
    }
  }

  // scales, quaternion, opacity
  double g_ls[3], g_q[4] = {0.0, 0.0, 0.0, 0.0}, g_o;
  double g_infl2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    g_ls[k] = g_S[k] * S[k];
    g_infl2 += g_S[k] * S[k] / (2.0 * infl2);
  }
  if (qvalid) {
    const double* G = g_R;
    double gq[4];
    gq[0] = 2.0 * (G[1] * qy + G[2] * qz + G[3] * qy - 2.0 * G[4] * qx - G[5] * qw + G[6] * qz + G[7] * qw -
                   2.0 * G[8] * qx);
    gq[1] = 2.0 * (-2.0 * G[0] * qy + G[1] * qx + G[2] * qw + G[3] * qx + G[5] * qz - G[6] * qw + G[7] * qz -
                   2.0 * G[8] * qy);
    gq[2] = 2.0 * (-2.0 * G[0] * qz - G[1] * qw + G[2] * qx + G[3] * qw - 2.0 * G[4] * qz + G[5] * qy + G[6] * qx +
                   G[7] * qy);
    gq[3] = 2.0 * (-G[1] * qz + G[2] * qy + G[3] * qz - G[5] * qx - G[6] * qy + G[7] * qx);
    const double dq = gq[0] * qx + gq[1] * qy + gq[2] * qz + gq[3] * qw;
#pragma unroll
    for (int k = 0; k < 4; k++) g_q[k] = (gq[k] - qn[k] * dq) / ql;
  }
  if (op_const) {
    g_o = g_infl2 * infl2 * (4.0 * op / (3.0 * 2.718281828459045)) * dop_do;
  } else {
    g_o = g_op * dop_do;
  }

  // colour: rgb = max(base + SH, 0) with SH (GpuShReader.apply), the base alone without
  if constexpr (K == 0) {
#pragma unroll
    for (int c = 0; c < 3; c++) col[c] = (float)g_rgb[c];
  } else {
    const int cap = min(p.max_sh_degree, DEG);
    const int kc = cap <= 0 ? 0 : (cap == 1 ? 3 : (cap == 2 ? 8 : (cap == 3 ? 15 : 24)));
    const double dx = cx - sd.origin[0], dy = cy - sd.origin[1], dz = cz - sd.origin[2];
    const double len = sqrt(dx * dx + dy * dy + dz * dz);
    const double inv = len > 0.0 ? 1.0 / len : 0.0;
    const double x = dx * inv, y = dy * inv, z = dz * inv;
    double Y[K], G[K][3];
    sh_basis_and_grad<K>(x, y, z, Y, G);
    const bool dir_ok = kc > 0 && len > 0.0;
    double sh[3] = {0.0, 0.0, 0.0};
    if (dir_ok) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (k < kc) {
#pragma unroll
          for (int c = 0; c < 3; c++) sh[c] = fma((double)col[3 + k * 3 + c], Y[k], sh[c]);
        }
      }
    }
    double gm[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      gm[c] = (double)col[c] + sh[c] > 0.0 ? g_rgb[c] : 0.0;
      col[c] = (float)gm[c];
    }
    double g_dir[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < K; k++) {
      const bool used = dir_ok && k < kc;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double value = (double)col[3 + k * 3 + c];  // read before the gradient takes its place
        col[3 + k * 3 + c] = used ? (float)(gm[c] * Y[k]) : 0.0f;
        if (used) {
          const double ck = gm[c] * value;
          g_dir[0] += ck * G[k][0];
          g_dir[1] += ck * G[k][1];
          g_dir[2] += ck * G[k][2];
        }
      }
    }
    if (dir_ok) {
      const double dd = g_dir[0] * x + g_dir[1] * y + g_dir[2] * z;
      g_c[0] += (g_dir[0] - x * dd) * inv;
      g_c[1] += (g_dir[1] - y * dd) * inv;
      g_c[2] += (g_dir[2] - z * dd) * inv;
    }
  }
  if (go_.centers) {
#pragma unroll
    for (int c = 0; c < 3; c++) go_.centers[i * 3 + c] = (float)g_c[c];
  }
  if (go_.log_scales) {
#pragma unroll
    for (int c = 0; c < 3; c++) go_.log_scales[i * 3 + c] = (float)g_ls[c];
  }
  if (go_.quats) reinterpret_cast<float4*>(go_.quats)[i] = make_float4((float)g_q[0], (float)g_q[1], (float)g_q[2], (float)g_q[3]);
  if (go_.opacities) go_.opacities[i] = (float)g_o;
}

constexpr int kBwdWarps = kBwdThreads / 32;
constexpr int kBwdQueue = 64;  // drawn rows waiting in a warp's queue

// Persistent warps over 32-row chunks: rows no eye drew get zero gradients at
// once (coalesced), drawn rows are queued and their gradients computed 32 at
// a time, so every lane of the float64 work is busy whatever the cull pattern.
template <int DEG, int CDT, int EYES>
__global__ void __launch_bounds__(kBwdThreads, kBwdBlocksPerSm) k_project_backward(const ProjDesc* __restrict__ descs,
                                                                  const GradsOut* __restrict__ grads, int n_desc,
                                                                  uint32_t total_chunks, GradsIn in) {
  constexpr int kRow = (1 + Coeffs<DEG>::value) * 3;
  constexpr int kPitch = kRow | 1;  // odd: a lane reading its own row hits its own banks
  __shared__ uint32_t s_row[kBwdWarps][kBwdQueue];
  __shared__ uint8_t s_drawn[kBwdWarps][kBwdQueue];
  __shared__ float s_col[kBwdWarps][32][kPitch];  // a batch's colour rows, then their gradients
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * kBwdWarps + (uint32_t)warp, nw = gridDim.x * kBwdWarps;
  int cur = -1, di = -1;
  uint32_t head = 0, queued = 0, chunk = gw;
  while (true) {
    const bool have = chunk < total_chunks;
    if (have && di < 0) {
      int d = 0;
      if (lane == 0) {
        int lo = 0, hi = n_desc - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (descs[mid].first_tile <= chunk) {
            lo = mid;
          } else {
            hi = mid - 1;
          }
        }
        d = lo;
      }
      di = __shfl_sync(0xffffffffu, d, 0);
    }
    // one site for the gradient: full batches, the rest before the object changes and at the end
    const uint32_t nb = queued >= 32 ? 32u : ((!have || di != cur) ? queued : 0u);
    if (nb) {
      // the batch's colour rows in by the whole warp (coalesced), the gradients out the same way
      const uint32_t q = (head + (uint32_t)lane) & (kBwdQueue - 1);
      const uint32_t my_row = (uint32_t)lane < nb ? s_row[warp][q] : 0u;
      const void* colors = descs[cur].table.colors;
      if constexpr (CDT == RDX_DTYPE_F16) {
#pragma unroll 8
        for (uint32_t r = 0; r < nb; r++) {
          const uint64_t row = __shfl_sync(0xffffffffu, my_row, (int)r);
          for (int e = lane; e < kRow; e += 32) s_col[warp][r][e] = (float)colour_value<DEG, CDT>(colors, row, e);
        }
      } else {
        // float32 rows copied asynchronously: every row's loads in flight at once
        for (uint32_t r = 0; r < nb; r++) {
          const uint64_t row = __shfl_sync(0xffffffffu, my_row, (int)r);
          const float* src = reinterpret_cast<const float*>(colors) + row * kRow;
          for (int e = lane; e < kRow; e += 32)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_col[warp][r][e])),
                         "l"(src + e)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
      }
      __syncwarp();
      if ((uint32_t)lane < nb) splat_backward<DEG, CDT, EYES>(descs[cur], grads[cur], in, my_row, s_drawn[warp][q], s_col[warp][lane]);
      __syncwarp();
      float* gcol = grads[cur].colors;
      if (gcol) {
        for (uint32_t r = 0; r < nb; r++) {
          const uint64_t row = __shfl_sync(0xffffffffu, my_row, (int)r);
          for (int e = lane; e < kRow; e += 32) gcol[row * kRow + e] = s_col[warp][r][e];
        }
      }
      __syncwarp();
      head = (head + nb) & (kBwdQueue - 1);
      queued -= nb;
      __syncwarp();
      continue;
    }
    if (!have) break;
    cur = di;
    const ProjDesc& sd = descs[cur];
    const uint64_t i = (uint64_t)(chunk - sd.first_tile) * kProjTile + (uint64_t)lane;
    const bool live = i < sd.count;
    uint32_t drawn = 0;
    if (live) {
      const uint64_t gi = sd.out_offset + i;
#pragma unroll
      for (int v = 0; v < EYES; v++)
        if (__ldg(in.fwd_opacity + (uint64_t)v * sd.out_n + gi) != 0.0f) drawn |= 1u << v;
      if (!drawn) {  // drawn by no eye: the outputs are constants
        const GradsOut go_ = grads[cur];
        if (go_.centers) go_.centers[i * 3] = go_.centers[i * 3 + 1] = go_.centers[i * 3 + 2] = 0.0f;
        if (go_.log_scales) go_.log_scales[i * 3] = go_.log_scales[i * 3 + 1] = go_.log_scales[i * 3 + 2] = 0.0f;
        if (go_.quats) reinterpret_cast<float4*>(go_.quats)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (go_.opacities) go_.opacities[i] = 0.0f;
      }
    }
    // colour rows of the undrawn live rows zeroed by the whole warp (coalesced)
    if (float* gcol = grads[cur].colors) {
      uint32_t undrawn = __ballot_sync(0xffffffffu, live && !drawn);
      const uint64_t i0 = (uint64_t)(chunk - sd.first_tile) * kProjTile;
      while (undrawn) {
        const int r = __ffs(undrawn) - 1;
        undrawn &= undrawn - 1u;
        for (int e = lane; e < kRow; e += 32) gcol[(i0 + (uint64_t)r) * kRow + e] = 0.0f;
      }
    }
    const uint32_t ballot = __ballot_sync(0xffffffffu, drawn != 0u);
    if (drawn) {
      const uint32_t q = (head + queued + (uint32_t)__popc(ballot & ((1u << lane) - 1u))) & (kBwdQueue - 1);
      s_row[warp][q] = (uint32_t)i;
      s_drawn[warp][q] = (uint8_t)drawn;
    }
    queued += (uint32_t)__popc(ballot);
    __syncwarp();
    chunk += nw;
    di = -1;
  }
}

using BwdKernel = void (*)(const ProjDesc*, const GradsOut*, int, uint32_t, GradsIn);

template <int DEG, int CDT>
BwdKernel pick_eyes(int eyes) {
  return eyes == 2 ? k_project_backward<DEG, CDT, 2> : k_project_backward<DEG, CDT, 1>;
}

template <int CDT>
BwdKernel pick_degree(int degree, int eyes) {
  switch (degree) {
    case 0: return pick_eyes<0, CDT>(eyes);
    case 1: return pick_eyes<1, CDT>(eyes);
    case 2: return pick_eyes<2, CDT>(eyes);
    case 3: return pick_eyes<3, CDT>(eyes);
    default: return pick_eyes<4, CDT>(eyes);
  }
}

}  // namespace

cudaError_t launch_project_backward(const ProjDesc* descs_dev, const GradsOut* grads_dev, const ProjDesc* descs_host,
                                    int n_desc, uint32_t total_chunks, const GradsIn& in, cudaStream_t stream) {
  if (total_chunks == 0 || n_desc == 0) return cudaSuccess;
  const ProjDesc& d0 = descs_host[0];
  const BwdKernel k = d0.table.color_dtype == RDX_DTYPE_F16 ? pick_degree<RDX_DTYPE_F16>(d0.table.sh_degree, d0.eyes)
                                                            : pick_degree<RDX_DTYPE_F32>(d0.table.sh_degree, d0.eyes);
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint32_t want = (total_chunks + kBwdWarps - 1) / kBwdWarps;
  const uint32_t blocks = min(want, (uint32_t)(sms * kBwdBlocksPerSm));
  k<<<blocks, kBwdThreads, 0, stream>>>(descs_dev, grads_dev, n_desc, total_chunks, in);
  return cudaGetLastError();
}

}  // namespace rdx
