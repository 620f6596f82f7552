/*
 * oracle.h - CPU FP64 restatement of the @sparkjsdev/radix per-frame splat
 * path (sort keys, stable sort, ext decoding, SH, ewa projection).
 *
 * TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared
 * against, and the timed CPU baseline. Nothing in the product links it.
 * Each function cites the reference file:line it restates (paths inside the
 * radix project).
 */
#ifndef RADIX_ORACLE_H
#define RADIX_ORACLE_H

#include <stdint.h>
#include "../include/radix_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* src/core/sort.ts:37-58 */
uint32_t orc_invalid_key(int bits);
uint32_t orc_valid_max(int bits);
uint32_t orc_sort_key(double distance, int bits);
/* src/gpu/sortKey.tsl.ts:17-26 */
uint32_t orc_sort_key_f32(float distance, int bits);
void orc_sort_keys(const double* distances, uint64_t n, int bits, uint32_t* keys);

/* src/core/sort.ts:64-163: returns 0, or -1 when ordering_len < count */
int orc_sort(const uint32_t* keys, uint64_t count, int bits, uint32_t* ordering,
             uint64_t ordering_len, uint32_t* visible);

/* src/core/encoding.ts:156-239, 21-112 */
double orc_decode_half(uint32_t h);
uint32_t orc_encode_half(double f);
void orc_decode_ext_rgb(uint32_t word, double rgb[3]);
uint32_t orc_encode_ext_rgb(const double rgb[3]);
void orc_decode_oct(uint32_t code, int bits, double out[3]);
uint32_t orc_encode_oct(const double v[3], int bits);
void orc_decode_quat_oct32(uint32_t code, double q[4]);
uint32_t orc_encode_quat_oct32(const double q[4]);
void orc_decode_quat_oct(uint32_t code, int axis_bits, int angle_bits, double q[4]);
uint32_t orc_encode_quat_oct(const double q[4], int axis_bits, int angle_bits);

/* src/core/sh.ts:362-407 */
void orc_sh_basis(const double dir[3], double out[24]);
void orc_sh_evaluate(const double* coeffs, const double dir[3], int degree, double out[3]);

/* The splat of a table row in object space (src/core/splats.ts:188-197 for ext) */
typedef struct orc_splat {
  double center[3];
  double scales[3];
  double quat[4];
  double opacity;
  double rgb[3];
  double sh[24 * 3];
  int sh_degree;
  double cov[6];      /* cov layout: xx, yy, zz, xy, xz, yz (then scales and quat are unused) */
  int has_cov;
} orc_splat;
void orc_load_splat(const rdx_table* table, uint64_t index, orc_splat* out);

/* Projection outputs in float64; any pointer may be NULL. Layouts as rdx_outputs. */
typedef struct orc_outputs {
  double* mean2d;
  double* conic;
  double* depth;
  double* opacity;
  double* rgb;
  double* radii;
  uint32_t* words;
  uint32_t* keys;
  double* distance;   /* [n] head-space distance */
  uint8_t* visible;   /* [E][n] 1 when the eye draws the splat */
} orc_outputs;

/*
 * projectCollection + SplatProjection.write + ewa.project
 * (SplatProjector.ts:106-194, SplatProjection.ts:131-153, projections.tsl.ts:95-148)
 * in float64. threads <= 0: all cores (OpenMP).
 */
int orc_project(const rdx_object* objects, int n_objects, const rdx_camera* camera,
                const rdx_params* params, int sort_bits, int cull_keys, int threads,
                const orc_outputs* out);

/*
 * The ray projection methods (projections.tsl.ts:170-474: rayProjection with
 * gutBound or htgsBound, and raygs) in float64: words [n][H + E * W] (head
 * words first, then each eye's; H, W = 6, 2 for 3dgut and htgs, 4, 3 for
 * raygs) and keys [n] (either may be NULL). Cov tables, and objects whose
 * object -> head matrix is not a rotation times a uniform scale, reach the
 * splat form through fromCov (the eigen decomposition of the head-space
 * covariance, src/gpu/splats.tsl.ts:189-199).
 */
#define ORC_METHOD_3DGUT 1
#define ORC_METHOD_HTGS 2
#define ORC_METHOD_RAYGS 3
int orc_project_rays(const rdx_object* objects, int n_objects, const rdx_camera* camera, const rdx_params* params,
                     int method, int sort_bits, int cull_keys, int threads, uint32_t* words, uint32_t* keys);

/* d(basis)/d(x, y, z) of the 24 basis functions above, as polynomials in x, y, z */
void orc_sh_basis_grad(const double dir[3], double out[24][3]);

/* Upstream gradients of a projection, laid out as orc_outputs (NULL: zero) */
typedef struct orc_grads_in {
  const double* mean2d;
  const double* conic;
  const double* depth;
  const double* opacity;
  const double* rgb;
} orc_grads_in;

/* Gradients of the collection's rows (raw tables): centers [n][3],
   log_scales [n][3], quats [n][4] (of the stored, unnormalised quaternion),
   opacities [n], colors [n][75] (base rgb, then the coefficients of bands
   1..4, coefficient-major RGB; beyond the table's degree: 0) */
typedef struct orc_grads_out {
  double* centers;
  double* log_scales;
  double* quats;
  double* opacities;
  double* colors;
} orc_grads_out;

/*
 * The analytic gradient of orc_project's mean2d, conic, depth, opacity and
 * rgb outputs (full pass) with respect to a raw table's fields, in float64.
 * An eye that culls a splat contributes nothing. Returns -1 for an ext table.
 */
int orc_project_backward(const rdx_object* objects, int n_objects, const rdx_camera* camera,
                         const rdx_params* params, const orc_grads_in* gin, const orc_grads_out* gout,
                         int threads);

/* Word codecs of the ewa projection (src/render/projection.tsl.ts:283-294) */
uint32_t orc_encode_depth20(double view_z);
uint32_t orc_encode_angle12(double angle);

/* A raw table encoded as Radix's ext layout (src/core/splats.ts:150-181 store
   path, src/core/sh.ts:114-135 ext SH), for fixtures of the ext reader */
int orc_encode_ext_table(const rdx_table* raw, uint32_t* ext_a, uint32_t* ext_b, uint32_t* const* ext_sh);

/* Fixtures: packedCodec.encode (src/core/splats.ts:279-286) and
   storeCovFields (splats.ts:236-243) of a raw table, and its SH coefficients
   in a codec (src/core/sh.ts:137-160), `stride` words per splat */
int orc_encode_packed_table(const rdx_table* raw, const float encoding[4], uint32_t* packed);
int orc_encode_cov_table(const rdx_table* raw, uint32_t* cov_a, uint32_t* cov_b);
int orc_sh_words(int codec, int degree);
int orc_encode_sh(const rdx_table* raw, int codec, uint32_t* words, int stride);

/* PlyFile.read (src/core/ply.ts:58-264) in float64 into raw-table columns
   (centers [n][3], log_scales [n][3], quats [n][4] normalised x y z w,
   opacities [n], colors [n][1 + K][3] of degree sh_degree, -1: the file's);
   the count, the file's SH degree and kind (0 standard, 1 point cloud,
   2 compressed) come back. -1 on a malformed file. */
int orc_ply_decode(const uint8_t* bytes, uint64_t nbytes, int sh_degree, double* centers, double* log_scales,
                   double* quats, double* opacities, double* colors, uint64_t* count, int* degree, int* kind);

/* SpzFile.read's per-splat decode (src/core/spz.ts:285-348) of an SPZ file's
   byte columns (a gzip payload's after its 16-byte header, or an NGSP file's
   decompressed streams) in float64 into raw-table columns: centers [n][3]
   (v1: halves; else 24-bit fixed point over 2^fractional_bits), log_scales
   [n][3] (byte / 16 - 10), quats [n][4] normalised x y z w (v3 and later:
   smallest three; else 3 bytes of x y z, w >= 0), opacities [n] (alpha / 255),
   colors [n][1 + K][3] of degree out_degree (base rgb (b / 255 - 0.5) SH_C0 /
   0.15 + 0.5, then (b - 128) / 128 coefficient-major). -1 on bad arguments. */
int orc_spz_decode(int version, uint64_t count, int sh_degree, int fractional_bits, const uint8_t* centers,
                   const uint8_t* alphas, const uint8_t* colors, const uint8_t* scales, const uint8_t* rotations,
                   const uint8_t* sh, int out_degree, double* out_centers, double* out_log_scales, double* out_quats,
                   double* out_opacities, double* out_colors);

/* The reference's defaults (src/render/splatParams.ts:68-72) */
void orc_params_default(rdx_params* p);

/* 4x4 column-major helpers (three.js Matrix4 semantics) */
void orc_mat4_mul(const double a[16], const double b[16], double out[16]);
int orc_mat4_invert(const double m[16], double out[16]);

#ifdef __cplusplus
}
#endif

#endif
