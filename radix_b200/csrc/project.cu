// Fused per-splat projection for sm_100a: table decode, SH colour from the
// head (object space), object -> head transform, ewa projection per eye, the
// reference's words, float outputs and the back-to-front sort key.
//
// Restates, fused: SplatProjector.build (src/render/SplatProjector.ts:153-194),
// SplatGenerator.fromSplats.withSh (src/gpu/splatGenerator.ts:152-158),
// GpuShReader.color/apply (src/gpu/sh.tsl.ts:255-266), transformCov
// (src/render/splatTransform.tsl.ts:120-140), prepareSplat / splatInView /
// culls (src/render/projection.tsl.ts:42-140), ewa.project
// (src/render/projections.tsl.ts:95-148) and SplatProjection.write
// (src/render/SplatProjection.ts:141-153).
//
// Structure: a persistent grid of independent warps; no block-wide barrier
// until the end. A warp walks 32-splat chunks. Phase 1 (a lane per splat):
// the centre, opacity and scales are read, the centre transformed in float64,
// the key distance and the centre culls computed; splats culled in every eye
// are finished there. The others go to a warp-private queue in shared memory
// (their SH rows and quaternions prefetched into L2). Whenever 32 are queued,
// phase 2 runs a lane per queued splat: SH, covariance and ewa. Culled splats'
// SH rows and quaternions are never read, and phase 2's lanes are all busy.
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

#include <map>
#include <mutex>
#include <utility>

#include "device_common.cuh"
#include "rdx_internal.h"
#include "table_rows.cuh"

namespace rdx {
namespace {

constexpr int kWarps = 4;  // warps per block of the launches that do not choose (the warps are independent)
constexpr int kChunk = kProjTile;      // splats per chunk (a warp's phase 1)
constexpr int kQueue = 64;             // candidate ring of a warp
static_assert(kChunk == 32, "a chunk is one warp wide");

// inSortGuard (projection.tsl.ts:145-155), cov form: whether splat i may show
// in the head's view widened by the guard. The head-space covariance's largest
// diagonal element and the reach in float64 with every operation explicitly
// rounded, in the oracle's order, so the guard's decisions (and the keys) are
// the oracle's. Only the kernels of launches with a guard hold this code: in
// the others, even unexecuted, it slowed every frame's projection by 5 %.
template <int LAYOUT>
__device__ __forceinline__ bool in_sort_guard(const ProjDesc& sd, uint64_t i, float opac, double ls0, double ls1,
                                           double ls2, double hx, double hy, double hz) {
  const DevParams& p = sd.params;
  const double ls[3] = {ls0, ls1, ls2};
  double inflate2 = 1.0;
  if (opac > 1.0f && p.lod_inflate) {
    const double o = fmin(dadd(dmul((double)opac, 4.0), -3.0), 5.0);
    const double inflate = pow(exp(__ddiv_rn(dadd(dmul(o, o), -1.0), 2.71828182845904523536)), 1.0 / 3.0);
    inflate2 = dmul(inflate, inflate);
  }
  double cv[9];  // object-space covariance, row-major
  if constexpr (LAYOUT == RDX_LAYOUT_COV) {
    double c6[6];
    load_cov(sd.table, i, c6);
    cv[0] = c6[0], cv[1] = c6[3], cv[2] = c6[4];
    cv[3] = c6[3], cv[4] = c6[1], cv[5] = c6[5];
    cv[6] = c6[4], cv[7] = c6[5], cv[8] = c6[2];
  } else {
    // M = R(q) diag(s) (math.tsl.ts:26-44), Sigma = M M^T
    double q[4];
    load_quat<LAYOUT>(sd.table, i, q);
    double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
    const double ql = __dsqrt_rn(dadd(dadd(dadd(dmul(qx, qx), dmul(qy, qy)), dmul(qz, qz)), dmul(qw, qw)));
    if (!(ql > 0.0)) {
      qx = qy = qz = 0.0;
      qw = 1.0;
    } else {
      qx = __ddiv_rn(qx, ql);
      qy = __ddiv_rn(qy, ql);
      qz = __ddiv_rn(qz, ql);
      qw = __ddiv_rn(qw, ql);
    }
    const double sx = exp(ls[0]), sy = exp(ls[1]), sz = exp(ls[2]);
    const double M[9] = {
        dmul(sx, dadd(1.0, -dmul(2.0, dadd(dmul(qy, qy), dmul(qz, qz))))),
        dmul(dmul(sy, 2.0), dadd(dmul(qx, qy), -dmul(qw, qz))),
        dmul(dmul(sz, 2.0), dadd(dmul(qx, qz), dmul(qw, qy))),
        dmul(dmul(sx, 2.0), dadd(dmul(qx, qy), dmul(qw, qz))),
        dmul(sy, dadd(1.0, -dmul(2.0, dadd(dmul(qx, qx), dmul(qz, qz))))),
        dmul(dmul(sz, 2.0), dadd(dmul(qy, qz), -dmul(qw, qx))),
        dmul(dmul(sx, 2.0), dadd(dmul(qx, qz), -dmul(qw, qy))),
        dmul(dmul(sy, 2.0), dadd(dmul(qy, qz), dmul(qw, qx))),
        dmul(sz, dadd(1.0, -dmul(2.0, dadd(dmul(qx, qx), dmul(qy, qy))))),
    };
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++)
        cv[r * 3 + c] = dadd(dadd(dmul(M[r * 3 + 0], M[c * 3 + 0]), dmul(M[r * 3 + 1], M[c * 3 + 1])),
                             dmul(M[r * 3 + 2], M[c * 3 + 2]));
  }
  // diag(A Sigma A^T) as (A Sigma) A^T, each sum left to right
  double ext2 = 0.0;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const double a0 = sd.a[r * 4 + 0], a1 = sd.a[r * 4 + 1], a2 = sd.a[r * 4 + 2];
    double t[3];
#pragma unroll
    for (int c = 0; c < 3; c++) t[c] = dadd(dadd(dmul(a0, cv[c]), dmul(a1, cv[3 + c])), dmul(a2, cv[6 + c]));
    const double v = dmul(dadd(dadd(dmul(t[0], a0), dmul(t[1], a1)), dmul(t[2], a2)), inflate2);
    ext2 = r == 0 ? v : fmax(ext2, v);
  }
  const double radius = dmul(__dsqrt_rn(ext2), (double)p.max_std_dev);
  const double* P = sd.eye[0].proj;
  const double clx = dadd(dadd(dadd(dmul(P[0], hx), dmul(P[4], hy)), dmul(P[8], hz)), P[12]);
  const double cly = dadd(dadd(dadd(dmul(P[1], hx), dmul(P[5], hy)), dmul(P[9], hz)), P[13]);
  const double clw = dadd(dadd(dadd(dmul(P[3], hx), dmul(P[7], hy)), dmul(P[11], hz)), P[15]);
  const double w = fmax(clw, 1e-6);
  const double rx = __ddiv_rn(dmul(P[0], radius), w), ry = __ddiv_rn(dmul(P[5], radius), w);
  const double edge = dadd((double)p.sort_guard, 1.0);
  const bool inside = dadd(fabs(__ddiv_rn(clx, w)), -rx) <= edge && dadd(fabs(__ddiv_rn(cly, w)), -ry) <= edge;
  const bool near_head = -hz <= radius;
  return hz < radius && (inside || near_head);
}

// A warp's shared memory: its descriptor and its candidate queue (a ring)
template <int EYES>
struct WarpSmem {
  ProjDesc desc;
  uint32_t idx[kQueue];    // row of the object
  uint32_t key[kQueue];    // the splat's valid key
  float c[3][kQueue];      // object-space centre
  uint32_t eye_ok[kQueue]; // eyes whose centre culls passed
  double e[EYES][6][kQueue];  // per eye: centre ex, ey, ez and clip x, y, w (float64)
};

// Kernel flavours: plain; with the sort guard's code (launches where an object
// sets a guard); host rows (raw tables whose colour rows may be pinned host
// memory read in place: a warp stages each batch's rows in shared memory with
// whole 16-byte pieces in row order, so a row crosses the bus in full requests
// instead of a lane's scattered ones)
constexpr int kPlain = 0, kGuarded = 1, kHostRows = 2;

// A warp's staged colour rows: 32 rows, each padded to an odd number of
// 16-byte pieces (a lane's reads of its row then fall in distinct banks)
template <int DEG, int VAR>
struct RowStage {
  static constexpr int kPieces = ColorRow<DEG, VAR>::kBytes / 16;
  static constexpr int kStride = kPieces | 1;
  static constexpr int kBytes = 32 * kStride * 16;
};

template <int LAYOUT, int DEG, int VAR, int EYES, int WPB, int FLAVOR>
__global__ void __launch_bounds__(WPB * 32) k_project(const ProjDesc* __restrict__ descs, int n_desc, uint32_t total_chunks,
                                                      ProjOutputs out) {
  constexpr bool GUARD = FLAVOR == kGuarded;
  constexpr bool HOST_ROWS = FLAVOR == kHostRows;
  static_assert(!HOST_ROWS || (WPB * sizeof(WarpSmem<EYES>)) % 16 == 0, "the staged rows start 16-byte aligned");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  WarpSmem<EYES>& W = reinterpret_cast<WarpSmem<EYES>*>(smem_raw)[warp];
  uint4* const rows = HOST_ROWS ? reinterpret_cast<uint4*>(smem_raw + WPB * sizeof(WarpSmem<EYES>) +
                                                           (size_t)warp * RowStage<DEG, VAR>::kBytes)
                                : nullptr;
  const ProjDesc& sd = W.desc;
  const uint32_t lt = (1u << lane) - 1u;

  pdl_trigger();  // the sort's first kernel may be placed now; it waits for this grid to complete
  if (blockIdx.x == 0 && out.zero) {
    for (uint64_t w = threadIdx.x; w < out.zero_words; w += blockDim.x) out.zero[w] = 0u;
  }

  int cur_desc = -1;
  uint32_t head = 0, queued = 0;

  // ---- phase 2: SH, covariance and ewa of nb queued splats (a lane each) ----
  auto process = [&](uint32_t nb) {
    const DevParams& p = sd.params;
    const bool busy = (uint32_t)lane < nb;
    const uint32_t q = (head + (uint32_t)lane) & (kQueue - 1);
    if constexpr (HOST_ROWS) {
      using RS = RowStage<DEG, VAR>;
      const uint4* colors = reinterpret_cast<const uint4*>(sd.table.colors);
      uint4 piece[RS::kPieces];
#pragma unroll
      for (int j = 0; j < RS::kPieces; j++) {
        const uint32_t f = (uint32_t)j * 32 + (uint32_t)lane;  // piece f of the batch: row f / kPieces
        const uint32_t r = f / RS::kPieces;
        if (r < nb) piece[j] = __ldg(colors + (uint64_t)W.idx[(head + r) & (kQueue - 1)] * RS::kPieces + (f - r * RS::kPieces));
      }
#pragma unroll
      for (int j = 0; j < RS::kPieces; j++) {
        const uint32_t f = (uint32_t)j * 32 + (uint32_t)lane;
        const uint32_t r = f / RS::kPieces;
        if (r < nb) rows[r * RS::kStride + (f - r * RS::kPieces)] = piece[j];
      }
      __syncwarp();
    }
    uint32_t key_out = invalid_key(sd.sort_bits);
    bool any_visible = false;
    if (busy) {
      const uint64_t i = W.idx[q];
      const uint64_t gi = sd.out_offset + i;
      float cf[3], opac;
      double ls[3];
      bool zero_cov;
      load_head<LAYOUT>(sd.table, i, cf, opac, ls, zero_cov);
      double rgb[3];
      colour<LAYOUT, DEG, VAR>(sd.table, i, (double)W.c[0][q] - sd.origin[0], (double)W.c[1][q] - sd.origin[1],
                               (double)W.c[2][q] - sd.origin[2], min(p.max_sh_degree, DEG), rgb,
                               HOST_ROWS ? rows + lane * RowStage<DEG, VAR>::kStride : nullptr);
      // prepareSplat (projection.tsl.ts:42-64), float64
      double op = opac, inflate2 = 1.0;
      if (op > 1.0) {
        op = fmin(op * 4.0 - 3.0, 5.0);
        if (p.lod_inflate) {
          inflate2 = exp((op * op - 1.0) * (2.0 / (3.0 * 2.718281828459045)));
          op = 1.0;
        }
      }
      const float std_dev = op > 1.0 ? (float)((double)p.max_std_dev + (op - 1.0) * 0.7) : p.max_std_dev;
      // scales^2 = exp(2 ln s) (the cov layout: the stored covariance), both times the LoD inflation
      double s2x = 0.0, s2y = 0.0, s2z = 0.0, cv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      double R[9] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
      if constexpr (LAYOUT == RDX_LAYOUT_COV) {
        load_cov(sd.table, i, cv);
#pragma unroll
        for (int k = 0; k < 6; k++) cv[k] *= inflate2;
      } else {
        s2x = exp(2.0 * ls[0]) * inflate2;
        s2y = exp(2.0 * ls[1]) * inflate2;
        s2z = exp(2.0 * ls[2]) * inflate2;
        double qv[4];
        load_quat<LAYOUT>(sd.table, i, qv);
        const double ql2 = qv[0] * qv[0] + qv[1] * qv[1] + qv[2] * qv[2] + qv[3] * qv[3];
        if (ql2 > 0.0) {
          const double qi = 1.0 / sqrt(ql2);
          qv[0] *= qi;
          qv[1] *= qi;
          qv[2] *= qi;
          qv[3] *= qi;
        } else {
          qv[0] = qv[1] = qv[2] = 0.0;
          qv[3] = 1.0;
        }
        const double qx = qv[0], qy = qv[1], qz = qv[2], qw = qv[3];
        // R(q), row-major (src/gpu/math.tsl.ts:26-44 without the scales)
        R[0] = 1.0 - 2.0 * (qy * qy + qz * qz);
        R[1] = 2.0 * (qx * qy - qw * qz);
        R[2] = 2.0 * (qx * qz + qw * qy);
        R[3] = 2.0 * (qx * qy + qw * qz);
        R[4] = 1.0 - 2.0 * (qx * qx + qz * qz);
        R[5] = 2.0 * (qy * qz - qw * qx);
        R[6] = 2.0 * (qx * qz - qw * qy);
        R[7] = 2.0 * (qy * qz + qw * qx);
        R[8] = 1.0 - 2.0 * (qx * qx + qy * qy);
      }
      const uint32_t eye_ok = W.eye_ok[q];
#pragma unroll
      for (int v = 0; v < EYES; v++) {
        const DevEye& e = sd.eye[v];
        const uint64_t ei = (uint64_t)v * sd.out_n + gi;
        bool ok = (eye_ok >> v) & 1u;
        const double ex = W.e[v][0][q], ey = W.e[v][1][q], ez = W.e[v][2][q];
        const double clx = W.e[v][3][q], cly = W.e[v][4][q], clw = W.e[v][5][q];
        // depth of field (projection.tsl.ts:117-125)
        double blur = p.blur_amount;
        const float fz = (float)ez;
        if (p.focal_distance > 0.0f && p.aperture_tan > 0.0f && ez < 0.0) {
          const double depth = -ez;
          const double coc_view = fabs(depth - (double)p.focal_distance) * (double)p.aperture_tan;
          const double focal_pixels = sd.height * 0.5 * e.proj[5];
          const double coc = e.ortho ? coc_view * focal_pixels : coc_view * focal_pixels / depth;
          blur = fmin(fmax(coc * coc, blur), (double)p.max_pixel_radius * p.max_pixel_radius);
        }
        double a_d = 0.0, b_d = 0.0, d_d = 0.0, det_d = 1.0, inv_det = 1.0, opacity_cd = 0.0;
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
          const double* Wm = e.wd;  // object -> eye 3x3
          const double w0x = j1x * Wm[0] + j2x * Wm[6], w0y = j1x * Wm[1] + j2x * Wm[7], w0z = j1x * Wm[2] + j2x * Wm[8];
          const double w1x = j1y * Wm[3] + j2y * Wm[6], w1y = j1y * Wm[4] + j2y * Wm[7], w1z = j1y * Wm[5] + j2y * Wm[8];
          double ra, rd, det_t;
          if constexpr (LAYOUT == RDX_LAYOUT_COV) {
            // cov2D = M Sigma M^T with the rows w0, w1 of M (float64: its det cancels less than float32 needs)
            const double sw0x = cv[0] * w0x + cv[3] * w0y + cv[4] * w0z;
            const double sw0y = cv[3] * w0x + cv[1] * w0y + cv[5] * w0z;
            const double sw0z = cv[4] * w0x + cv[5] * w0y + cv[2] * w0z;
            const double sw1x = cv[0] * w1x + cv[3] * w1y + cv[4] * w1z;
            const double sw1y = cv[3] * w1x + cv[1] * w1y + cv[5] * w1z;
            const double sw1z = cv[4] * w1x + cv[5] * w1y + cv[2] * w1z;
            ra = w0x * sw0x + w0y * sw0y + w0z * sw0z;
            rd = w1x * sw1x + w1y * sw1y + w1z * sw1z;
            b_d = w0x * sw1x + w0y * sw1y + w0z * sw1z;
            det_t = ra * rd - b_d * b_d;
          } else {
            const double u00 = w0x * R[0] + w0y * R[3] + w0z * R[6];
            const double u01 = w0x * R[1] + w0y * R[4] + w0z * R[7];
            const double u02 = w0x * R[2] + w0y * R[5] + w0z * R[8];
            const double u10 = w1x * R[0] + w1y * R[3] + w1z * R[6];
            const double u11 = w1x * R[1] + w1y * R[4] + w1z * R[7];
            const double u12 = w1x * R[2] + w1y * R[5] + w1z * R[8];
            ra = u00 * u00 * s2x + u01 * u01 * s2y + u02 * u02 * s2z;
            rd = u10 * u10 * s2x + u11 * u11 * s2y + u12 * u12 * s2z;
            b_d = u00 * u10 * s2x + u01 * u11 * s2y + u02 * u12 * s2z;
            const double m0 = u01 * u12 - u02 * u11;
            const double m1 = u02 * u10 - u00 * u12;
            const double m2 = u00 * u11 - u01 * u10;
            det_t = m0 * m0 * (s2y * s2z) + m1 * m1 * (s2x * s2z) + m2 * m2 * (s2x * s2y);
          }
          const double pre = p.pre_blur_amount, full = (double)p.pre_blur_amount + blur;
          const double det_orig = det_t + pre * (ra + rd) + pre * pre;
          det_d = det_t + full * (ra + rd) + full * full;
          a_d = ra + full;
          d_d = rd + full;
          inv_det = 1.0 / det_d;
          opacity_cd = op * sqrt(fmax(0.0, det_orig * inv_det));
          // contribution >= minContribution holds for any non-NaN value when the bound is <= 0, and a NaN
          // opacity already fails the minAlpha test: the square root is needed only for a positive bound
          const bool contributes =
              p.min_contribution <= 0.0f ||
              opacity_cd * 6.283185307179586 * sqrt(fmax(0.0, det_d)) >= (double)p.min_contribution;
          // boundFromCov (projection.tsl.ts:223-240)
          const float a = (float)a_d, b = (float)b_d, d = (float)d_d, det = (float)det_d;
          const float half = (a - d) * 0.5f;
          const float eigen1 = (a + d) * 0.5f + sqrtf(half * half + b * b);
          const float eigen2 = eigen1 > 0.0f ? fmaxf(det / eigen1, 0.0f) : 0.0f;
          scale1 = fminf(p.max_pixel_radius, std_dev * sqrtf(fmaxf(eigen1, 0.0f)));
          scale2 = fminf(p.max_pixel_radius, std_dev * sqrtf(eigen2));
          const bool bound_ok = scale1 >= p.min_pixel_radius || scale2 >= p.min_pixel_radius;
          if (bound_ok && (out.radii || out.words)) {  // the angle is an output of the words and radii only
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
          ok = opacity_cd >= (double)p.min_alpha && contributes && bound_ok;
        }
        if (ok) {
          const double inv_w = 1.0 / clw;
          const double ndcx = clx * inv_w, ndcy = cly * inv_w;
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
      // SplatProjection.write (SplatProjection.ts:150-151): culled in every eye -> invalid
      if (sd.cull_keys) {
        key_out = any_visible ? W.key[q] : invalid_key(sd.sort_bits);
        if (out.keys) out.keys[gi] = key_out;
      }
    }
    head = (head + nb) & (kQueue - 1);
    queued -= nb;
    __syncwarp();
  };

  const uint32_t gw = blockIdx.x * WPB + (uint32_t)warp;
  const uint32_t nw = gridDim.x * WPB;
  // One loop with a single site for each phase keeps the kernel's code small
  // (phase 2 is large; inlined at several sites it thrashes the instruction
  // cache). Each turn either runs phase 2 on a batch of queued splats or
  // phase 1 on the next chunk.
  uint32_t chunk = gw;
  int di = -1;  // descriptor of `chunk` (-1: not looked up yet)
  while (true) {
    const bool have_chunk = chunk < total_chunks;
    if (have_chunk && di < 0) {
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
    // full batches; the rest before the object changes (the queue holds one object's splats) and at the end
    const bool switching = !have_chunk || di != cur_desc;
    const uint32_t nb = queued >= 32 ? 32u : (switching ? queued : 0u);
    if (nb) {
      process(nb);
      continue;
    }
    if (!have_chunk) break;
    if (di != cur_desc) {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&descs[di]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&W.desc);
      for (int w = lane; w < (int)(sizeof(ProjDesc) / 4); w += 32) dst[w] = src[w];
      __syncwarp();
      cur_desc = di;
    }
    const DevParams& p = sd.params;
    // keys only: culled splats keep their keys (SplatProjection.ts:150-151 applies to a full projection)
    const bool cull_keys = sd.cull_keys && !sd.keys_only;
    const uint64_t i0 = (uint64_t)(chunk - sd.first_tile) * kChunk;
    const uint64_t i = i0 + (uint64_t)lane;
    const uint64_t gi = sd.out_offset + i;
#ifdef RDX_CHECK
    // a row of the object whose outputs would fall past the launch's (a planning error)
    const bool outside = i < sd.count && gi >= sd.out_n;
    if (outside) check_failed(out.check_flag);
    const bool live = i < sd.count && !outside;
#else
    const bool live = i < sd.count;
#endif
    if (i0 + (uint64_t)nw * kChunk < sd.count) prefetch_head<LAYOUT>(sd.table, i0 + (uint64_t)nw * kChunk, sd.count, lane);

    // ---- phase 1: centre, distance, centre culls ----
    bool candidate = false;
    uint32_t key = invalid_key(sd.sort_bits), kv = 0, eye_ok = 0;
    float cf[3] = {0.f, 0.f, 0.f};
    double pe[EYES][6];
    if (live) {
      float opac;
      double ls[3];
      bool zero_cov;
      load_head<LAYOUT>(sd.table, i, cf, opac, ls, zero_cov);
      const double cx = cf[0], cy = cf[1], cz = cf[2];
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
      const bool degenerate = sd.degenerate || zero_cov;
      const bool invisible = op <= 0.0 || op < (double)p.min_alpha || degenerate;
      bool guarded = true;
      // inSortGuard (off by default): compiled into the guard's kernels only
      if constexpr (GUARD) {
        if (p.sort_guard > 0.0f && !invisible) guarded = in_sort_guard<LAYOUT>(sd, i, opac, ls[0], ls[1], ls[2], hx, hy, hz);
      }
      kv = key_of_bits(__float_as_uint(__double2float_rn(distance)), sd.sort_bits);
      if (!cull_keys && !invisible && guarded) key = kv;
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
          if (!culled) eye_ok |= 1u << v;
          pe[v][0] = ex;
          pe[v][1] = ey;
          pe[v][2] = ez;
          pe[v][3] = clx;
          pe[v][4] = cly;
          pe[v][5] = clw;
        }
      }
      candidate = eye_ok != 0;
      if (candidate) {
        if constexpr (HOST_ROWS) {
          prefetch_l2(sd.table.quats + i * 4);
        } else {
          prefetch_rows<LAYOUT, DEG, VAR>(sd.table, i);
        }
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
    // keys known now: every key without cullKeys, culled splats' with it
    const bool key_final = live && (!cull_keys || !candidate);
    if (key_final && out.keys) out.keys[gi] = key;
    // enqueue the candidates, in row order
    const uint32_t ballot = __ballot_sync(0xffffffffu, candidate);
    // their rows of host columns read in place cross the bus: counted once a chunk
    if (sd.host_row_bytes && lane == 0 && ballot && out.host_bytes)
      atomicAdd(out.host_bytes, (unsigned long long)__popc(ballot) * sd.host_row_bytes);
    if (candidate) {
      const uint32_t q = (head + queued + (uint32_t)__popc(ballot & lt)) & (kQueue - 1);
      W.idx[q] = (uint32_t)i;
      W.key[q] = kv;
      W.c[0][q] = cf[0];
      W.c[1][q] = cf[1];
      W.c[2][q] = cf[2];
      W.eye_ok[q] = eye_ok;
#pragma unroll
      for (int v = 0; v < EYES; v++) {
#pragma unroll
        for (int f = 0; f < 6; f++) W.e[v][f][q] = pe[v][f];
      }
    }
    queued += (uint32_t)__popc(ballot);
    __syncwarp();
    chunk += nw;
    di = -1;
  }
}

using ProjKernel = void (*)(const ProjDesc*, int, uint32_t, ProjOutputs);

struct Picked {
  ProjKernel fn;
  int smem;   // per block
  int warps;  // per block
};

// Raw tables (the benchmark's) may launch with 2, 4 or 8 warps per block; the
// other layouts, and every launch with a sort guard, with 4
// Raw SH-3 tables (the benchmark's) also have the host-rows flavour (4-warp
// blocks): their rows are whole 16-byte pieces
template <int LAYOUT, int DEG, int VAR>
constexpr bool kHasHostRows = LAYOUT == RDX_LAYOUT_RAW && DEG == 3 && ColorRow<DEG, VAR>::kBytes % 16 == 0;

template <int LAYOUT, int DEG, int VAR, int EYES>
Picked picked(int warps, bool guard, bool host_rows) {
  constexpr int kSmem = (int)sizeof(WarpSmem<EYES>);
  if (guard) return {k_project<LAYOUT, DEG, VAR, EYES, kWarps, kGuarded>, kWarps * kSmem, kWarps};
  if constexpr (kHasHostRows<LAYOUT, DEG, VAR>) {
    if (host_rows) {
      constexpr int kStage = RowStage<DEG, VAR>::kBytes;
      return {k_project<LAYOUT, DEG, VAR, EYES, kWarps, kHostRows>, kWarps * (kSmem + kStage), kWarps};
    }
  }
  if constexpr (LAYOUT == RDX_LAYOUT_RAW) {
    if (warps == 2) return {k_project<LAYOUT, DEG, VAR, EYES, 2, kPlain>, 2 * kSmem, 2};
    if (warps == 8) return {k_project<LAYOUT, DEG, VAR, EYES, 8, kPlain>, 8 * kSmem, 8};
  }
  return {k_project<LAYOUT, DEG, VAR, EYES, kWarps, kPlain>, kWarps * kSmem, kWarps};
}

template <int LAYOUT, int DEG, int VAR>
Picked pick_eyes(int eyes, int warps, bool guard, bool host_rows) {
  return eyes == 2 ? picked<LAYOUT, DEG, VAR, 2>(warps, guard, host_rows)
                   : picked<LAYOUT, DEG, VAR, 1>(warps, guard, host_rows);
}

template <int LAYOUT, int VAR>
Picked pick_degree(int degree, int eyes, int warps, bool guard, bool host_rows) {
  switch (degree) {
    case 0: return pick_eyes<LAYOUT, 0, VAR>(eyes, warps, guard, host_rows);
    case 1: return pick_eyes<LAYOUT, 1, VAR>(eyes, warps, guard, host_rows);
    case 2: return pick_eyes<LAYOUT, 2, VAR>(eyes, warps, guard, host_rows);
    case 3: return pick_eyes<LAYOUT, 3, VAR>(eyes, warps, guard, host_rows);
    default: return pick_eyes<LAYOUT, 4, VAR>(eyes, warps, guard, host_rows);
  }
}

template <int LAYOUT>
Picked pick_codec(int degree, int codec, int eyes, int warps, bool guard) {
  // without SH the codec is immaterial: one kernel
  if (codec == RDX_SH_PACKED && degree > 0) return pick_degree<LAYOUT, RDX_SH_PACKED>(degree, eyes, warps, guard, false);
  return pick_degree<LAYOUT, RDX_SH_EXT>(degree, eyes, warps, guard, false);
}

Picked pick_kernel(const DevTable& t, int eyes, int warps, bool guard, bool host_rows) {
  switch (t.layout) {
    case RDX_LAYOUT_EXT: return pick_codec<RDX_LAYOUT_EXT>(t.sh_degree, t.sh_codec, eyes, warps, guard);
    case RDX_LAYOUT_PACKED: return pick_codec<RDX_LAYOUT_PACKED>(t.sh_degree, t.sh_codec, eyes, warps, guard);
    case RDX_LAYOUT_COV: return pick_codec<RDX_LAYOUT_COV>(t.sh_degree, t.sh_codec, eyes, warps, guard);
    default:
      if (t.color_dtype == RDX_DTYPE_F16)
        return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F16>(t.sh_degree, eyes, warps, guard, host_rows);
      return pick_degree<RDX_LAYOUT_RAW, RDX_DTYPE_F32>(t.sh_degree, eyes, warps, guard, host_rows);
  }
}

// Resident blocks of one projection kernel on the current device, found once
// (with its shared-memory attribute set) and kept: a launch then makes no
// attribute or occupancy query
int resident_blocks(const Picked& k, cudaError_t* err) {
  static std::mutex mu;
  static std::map<std::pair<int, ProjKernel>, int> cache;
  int device = 0;
  *err = cudaGetDevice(&device);
  if (*err != cudaSuccess) return 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({device, k.fn});
    if (it != cache.end()) return it->second;
  }
  int sms = 0, per_sm = 0;
  *err = cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem);
  if (*err != cudaSuccess) return 0;
  *err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (*err != cudaSuccess) return 0;
  *err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.warps * 32, k.smem);
  if (*err != cudaSuccess) return 0;
  const int blocks = sms * (per_sm < 1 ? 1 : per_sm);
  std::lock_guard<std::mutex> lock(mu);
  cache[{device, k.fn}] = blocks;
  return blocks;
}

}  // namespace

int project_warps_supported(int warps) { return warps == 2 || warps == 4 || warps == 8; }

bool project_host_rows_supported(const DevTable& t) {
  if (t.layout != RDX_LAYOUT_RAW || t.sh_degree != 3) return false;
  return t.color_dtype == RDX_DTYPE_F16 ? kHasHostRows<RDX_LAYOUT_RAW, 3, RDX_DTYPE_F16>
                                        : kHasHostRows<RDX_LAYOUT_RAW, 3, RDX_DTYPE_F32>;
}

cudaError_t launch_project(const ProjDesc* descs_dev, const ProjDesc* descs_host, int n_desc, uint32_t total_chunks,
                           const ProjOutputs& out, uint32_t* error_flag, cudaStream_t stream, int warps) {
  if (total_chunks == 0 || n_desc == 0) return cudaSuccess;
  ProjOutputs outs = out;
  outs.check_flag = error_flag;  // no device wait in this kernel: the word records only clamped rows
  if (warps == 0) warps = kWarps;
  if (!project_warps_supported(warps)) return cudaErrorInvalidValue;
  // One kernel per launch: the caller groups objects by table kind
  const ProjDesc& d0 = descs_host[0];
  bool guard = false;  // an object of the launch keys its splats through the sort guard
  bool host_rows = false;  // an object's colour rows are read from host memory in place
  for (int j = 0; j < n_desc; j++) {
    guard = guard || descs_host[j].params.sort_guard > 0.0f;
    host_rows = host_rows || descs_host[j].host_row_bytes > 0;
  }
  if (host_rows && guard) return cudaErrorInvalidValue;  // the caller copies the rows of guarded launches
  const Picked k = pick_kernel(d0.table, d0.eyes, warps, guard, host_rows);
  cudaError_t err = cudaSuccess;
  const int blocks = resident_blocks(k, &err);
  if (err != cudaSuccess) return err;
  const uint32_t want = (total_chunks + (uint32_t)k.warps - 1) / (uint32_t)k.warps;
  const uint32_t grid = min(want, (uint32_t)blocks);
  k.fn<<<grid, k.warps * 32, k.smem, stream>>>(descs_dev, n_desc, total_chunks, outs);
  return cudaGetLastError();
}

}  // namespace rdx
