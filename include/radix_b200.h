/*
 * radix_b200.h - C ABI of the B200 (sm_100a) splat pipeline: back-to-front
 * sort keys, a stable onesweep radix sort of keys and indices, EWA projection
 * of 3D covariances to 2D conics, and spherical-harmonic colour (bands 1-4
 * over the base colour).
 *
 * Every entry point replaces one interface of @sparkjsdev/radix (paths below
 * are inside that project). All pointers are plain C pointers. A pointer may
 * address device memory (cudaMalloc / torch) or host memory; host buffers are
 * staged through the context's device buffers, and a call that touches host
 * memory returns only after its results are in place. A call on device memory
 * only returns after enqueueing its kernels on the context's stream.
 *
 * Matrices are 4x4, float64, column-major (element (row r, column c) at
 * [c * 4 + r]): the order of three.js Matrix4.elements.
 *
 * Errors: every call returns an RDX_* status; rdx_last_error() gives the
 * message of the last failure on that context (the reference's Error texts
 * where it has one).
 */
#ifndef RADIX_B200_H
#define RADIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RDX_VERSION 1

#define RDX_OK 0
#define RDX_ERR_ARG 1          /* invalid argument (bad bits, null pointer, ...) */
#define RDX_ERR_CAPACITY 2     /* an output too small, or a size above a limit */
#define RDX_ERR_CUDA 3         /* a CUDA runtime error */
#define RDX_ERR_TIMEOUT 4      /* a bounded device wait gave up (lookback) */
#define RDX_ERR_UNSUPPORTED 5  /* a layout / degree / option this build lacks */
#define RDX_ERR_NOMEM 6        /* device or pinned host allocation failed */

/* Splat table layouts */
#define RDX_LAYOUT_RAW 0     /* float32 columns (3DGS parameters) */
#define RDX_LAYOUT_EXT 1     /* Radix extSplats (2 x uint32x4) */
#define RDX_LAYOUT_PACKED 2  /* Radix packedSplats (uint32x4) */
#define RDX_LAYOUT_COV 3     /* Radix covSplats (2 x uint32x4) */

/* SH codecs of the ext / packed / cov layouts (src/core/sh.ts:13-24) */
#define RDX_SH_EXT 0     /* one ext rgb word per coefficient */
#define RDX_SH_PACKED 1  /* per band a scale byte, then a sint8 per value */

/* Element types of a raw table's colour block */
#define RDX_DTYPE_F32 0
#define RDX_DTYPE_F16 1

/* Projection passes (SplatProjector.ts ProjectPass) */
#define RDX_PASS_FULL 0 /* words / float outputs and keys */
#define RDX_PASS_KEYS 1 /* keys only (the CPU-sort pass, SplatProjection.writeKeys) */

typedef struct rdx_ctx rdx_ctx;

/*
 * One splat table.
 *
 * RDX_LAYOUT_RAW: columns of `count` rows
 *   centers      float32 [count][3]
 *   log_scales   float32 [count][3]   (scale = exp(log_scale))
 *   quats        float32 [count][4]   (x, y, z, w; normalised on use)
 *   opacities    float32 [count]      (1 = opaque; above 1 = LoD stretch)
 *   colors       [count][1 + K][3] of color_dtype: the base rgb (band 0),
 *                then K = 3 / 8 / 15 / 24 SH coefficients of bands
 *                1..sh_degree, coefficient-major RGB (src/core/sh.ts:7-11).
 *   Rows of colors must start 4-byte aligned; other columns as their type.
 *
 * RDX_LAYOUT_EXT / RDX_LAYOUT_COV: Radix's ArrayData columns, drop-in
 *   ext_a, ext_b uint32 [count][4]    extA / extB, or covA / covB
 *                (src/core/splats.ts:10-32)
 * RDX_LAYOUT_PACKED:
 *   packed       uint32 [count][4]    (src/core/splats.ts:28-32)
 *   packed_encoding  rgbMin, rgbMax, lnScaleMin, lnScaleMax (the bundle's
 *                meta.encoding; defaults 0, 1, -12, 9)
 * SH of these layouts, in codec sh_codec (src/core/sh.ts:13-24):
 *   ext_sh[t]    uint32 [count][4]    per-splat texel channel t (<codec>ShA,
 *                <codec>ShB, ...), or, when sh_palette is set,
 *   sh_palette   uint32 [entries * sh_stride][4]  an ShPalette's shEntries,
 *   sh_label     uint16 [count]       each splat's entry (labels past
 *                sh_palette_size read the last entry).
 */
typedef struct rdx_table {
  int32_t layout;      /* RDX_LAYOUT_* */
  int32_t sh_degree;   /* 0..4: SH bands stored above the base colour */
  int32_t color_dtype; /* raw only: RDX_DTYPE_F32 or RDX_DTYPE_F16 */
  int32_t sh_codec;    /* ext / packed / cov: RDX_SH_EXT or RDX_SH_PACKED */
  uint64_t count;
  const float* centers;
  const float* log_scales;
  const float* quats;
  const float* opacities;
  const void* colors;
  const uint32_t* ext_a;
  const uint32_t* ext_b;
  const uint32_t* ext_sh[6];
  const uint32_t* packed;
  float packed_encoding[4];
  const uint32_t* sh_palette;
  const uint16_t* sh_label;
  uint32_t sh_stride;        /* texels per palette entry */
  uint32_t sh_palette_size;  /* palette entries */
} rdx_table;

/*
 * Projection parameters: SplatViewParams + SplatObjectParams
 * (src/render/splatParams.ts:8-43), defaults from rdx_params_default
 * (splatParams.ts:68-72).
 */
typedef struct rdx_params {
  float max_std_dev;      /* sqrt(8) */
  float min_alpha;        /* 0.5 / 255 */
  float falloff;          /* 1 (read by the draw only) */
  int32_t lod_inflate;    /* 1 */
  float blur_amount;      /* 0.3 px^2 */
  float pre_blur_amount;  /* 0 */
  float clip_xy;          /* 1.4 */
  float min_pixel_radius; /* 0 */
  float max_pixel_radius; /* 512 */
  float min_contribution; /* 0 */
  float focal_distance;   /* 0 */
  float aperture_tan;     /* 0 */
  float sort_guard;       /* 0 */
  int32_t max_sh_degree;  /* 4 */
} rdx_params;

/* One eye: world -> eye (camera.matrixWorldInverse) and its projection */
typedef struct rdx_eye {
  double view[16];
  double projection[16];
  int32_t ortho;
  int32_t reserved;
} rdx_eye;

/*
 * The camera of one render (SplatCamera.setViews, src/render/splatCamera.ts:
 * 119-138): world -> head, 1 or 2 eyes sharing one render size, and the NDC
 * depth of the near plane (0: WebGPU clip convention, -1: WebGL).
 */
typedef struct rdx_camera {
  double head[16];
  int32_t eyes;
  int32_t reserved;
  rdx_eye eye[2];
  double width;
  double height;
  double ndc_z_min;
} rdx_camera;

/*
 * One splat object of a collection (SplatCollection.ts:54-65): `count` splats
 * of `table` drawn with `world` (object -> world). Projected splat i of the
 * collection is splat i - offset of the object holding it; offsets are the
 * running sum of counts in object order. `params` overrides the call's params
 * for this object (NULL: the call's).
 */
typedef struct rdx_object {
  const rdx_table* table;
  uint64_t count;
  double world[16];
  const rdx_params* params;
} rdx_object;

/*
 * Projection outputs; any pointer may be NULL (not written). E = eyes,
 * n = splats of the collection. A culled eye writes zeros (opacity 0), as the
 * reference marks a culled eye by a zero opacity byte.
 *   mean2d   float32 [E][n][2]  pixels, (ndc + 1) / 2 * size (y up, as NDC)
 *   conic    float32 [E][n][3]  inverse of the blurred 2D covariance
 *                               (a, b, d) in px^2: (d, -b, a) / det
 *   depth    float32 [E][n]     -z in the eye
 *   opacity  float32 [E][n]     opacity after the blur compensation
 *   rgb      float32 [E][n][3]  base colour + SH from the head, clamped at 0
 *   radii    float32 [E][n][3]  bound half extents (px) and angle [0, pi)
 *   words    uint32  [n][4E]    the ewa words per eye (projections.tsl.ts:
 *                               135-140): ndc 2x16; depth20 | angle12 << 20;
 *                               ext rgb; opacity8 | 2 x 12-bit log2 scales
 *   keys     uint32  [n]        sort keys (SplatProjection.ts:141-153)
 */
typedef struct rdx_outputs {
  float* mean2d;
  float* conic;
  float* depth;
  float* opacity;
  float* rgb;
  float* radii;
  uint32_t* words;
  uint32_t* keys;
} rdx_outputs;

/* ---- context ---- */

/* A context on CUDA device `device`: its stream, scratch and error state. */
int rdx_ctx_create(int device, rdx_ctx** out);
int rdx_ctx_destroy(rdx_ctx* ctx);
/* Run on `stream` (a cudaStream_t, cudaStreamLegacy included; NULL: the context's own stream). */
int rdx_ctx_set_stream(rdx_ctx* ctx, void* stream);
/* Wait for the context's stream; reports a device-side timeout flag. */
int rdx_ctx_synchronize(rdx_ctx* ctx);
/* Grow scratch for sorts of up to max_keys keys, so later calls allocate nothing. */
int rdx_ctx_reserve(rdx_ctx* ctx, uint64_t max_keys);
/* Text of the context's last error ("" when none). */
const char* rdx_last_error(const rdx_ctx* ctx);
int rdx_version(void);

/*
 * Phase timing, after the reference's GpuProfiler phases (src/gpu/GpuProfiler.ts:
 * 1-57, SplatRenderer.ts:141-142, 426-437): with profiling on, calls record CUDA
 * events around each phase on the context's stream. rdx_ctx_phase_times waits
 * for the stream and returns, per phase, the summed milliseconds and the number
 * of timed runs since the last read, then clears them.
 */
#define RDX_PHASE_PROJECT 0 /* the fused projection kernel(s); the gradient and file decode kernels */
#define RDX_PHASE_SORT 1    /* histogram + onesweep passes (+ compaction) */
#define RDX_PHASE_COPY_IN 2 /* host -> device staging */
#define RDX_PHASE_COPY_OUT 3
#define RDX_PHASE_BATCH 4   /* one replay of a batch's CUDA graph */
#define RDX_PHASES 5
int rdx_ctx_set_profiling(rdx_ctx* ctx, int on);
int rdx_ctx_phase_times(rdx_ctx* ctx, double* ms, uint64_t* runs);
/*
 * Bounded device waits of this context's sorts. `polls`: how often a wait on
 * another tile's lookback word is polled before it gives up, sets the
 * context's error flag and lets its kernel finish (0: 2^22, the default);
 * the call that synchronises (or rdx_ctx_synchronize) then returns
 * RDX_ERR_TIMEOUT, and the context stays usable. `silent_pass` >= 0 is a test
 * hook: in the next sort only, the first tile of that digit pass publishes no
 * lookback word, so its successors' waits run out. A batch takes `polls` when
 * it is created. No counterpart in the reference, whose sorts throw on
 * misuse (WgpuRadixSort.ts:150-152) and have no device waits.
 */
int rdx_ctx_set_wait(rdx_ctx* ctx, uint32_t polls, int silent_pass);
/*
 * How this context's sorts run their digit passes (every variant gives the
 * same order): -1 a choice of rdx_batch_tune / rdx_sort_tune for the
 * workload's shape, else variant 0 (the default); 0 one onesweep kernel per
 * pass, 1024-key tiles for sorts of at most 1M keys and 4096-key tiles above;
 * 1-3 one cooperative kernel for every pass of a one-segment sort (1: 1024
 * threads x 16 keys per block, 2: 512 x 16, 3: 1024 x 8); 4-6 onesweep
 * passes in 4096-, 2048- or 1024-key tiles. A variant a sort cannot take
 * (cooperative with several segments, tiles its lookback words do not hold)
 * falls back to 0's tiles. A batch takes the choice when it is created. The
 * reference's radix sort has one such knob, keysPerThread 8 or 16
 * (WgpuRadixSort.ts:80-91).
 */
int rdx_ctx_set_sort_variant(rdx_ctx* ctx, int variant);

/* Kernels this context has launched since it was created. */
int rdx_ctx_launches(rdx_ctx* ctx, uint64_t* launches);

/*
 * How frame and projection calls read tables in host memory.
 * RDX_HOST_IN_PLACE (the default): the colour rows of a raw SH-3 table (the
 * largest column, which only drawn candidates read) are read by the
 * projection kernel in place when they are pinned host memory mapped into the
 * device's address space: a warp stages each batch of 32 candidates' rows in
 * whole 16-byte pieces, so only the rows of splats that pass the centre culls
 * cross the bus, in full requests. Every other host column (and pageable
 * memory, and every column of a call with a sort guard) is copied in before
 * the projection. RDX_HOST_COPY: every host column is copied in. In place
 * moves fewer bytes when the view culls splats; with every splat in view the
 * copy is a little faster. Either way the call returns once the device is
 * done with the host columns.
 */
#define RDX_HOST_COPY 0
#define RDX_HOST_IN_PLACE 1
int rdx_ctx_set_host_reads(rdx_ctx* ctx, int mode);
/* Bytes of table columns that frame and projection calls moved from host
 * memory (copies, and rows read in place) since the last query; waits for the
 * context's stream. */
int rdx_ctx_host_bytes(rdx_ctx* ctx, uint64_t* bytes);

/* Fill `p` with the reference's defaults (splatParams.ts:68-72). */
void rdx_params_default(rdx_params* p);

/* ---- sort keys ---- */

/*
 * SortKeys.compute (src/core/sort.ts:46-58) for n float64 distances: the
 * distance rounded to float32, non-finite -> the invalid key 2^bits - 1,
 * else min(mask ^ q, validMax).
 */
int rdx_sort_keys_compute(rdx_ctx* ctx, const double* distances, uint64_t n, int bits, uint32_t* keys);
/* GpuSortKeys.compute (src/gpu/sortKey.tsl.ts:17-26): float32 distances, max(d, 0). */
int rdx_sort_keys_compute_f32(rdx_ctx* ctx, const float* distances, uint64_t n, int bits, uint32_t* keys);

/* ---- sorting ---- */

/*
 * SortKeys.sort (src/core/sort.ts:64-82): the stable ascending order of the
 * first `count` keys as indices into `ordering` (ordering_len >= count, else
 * RDX_ERR_CAPACITY with the reference's message; entries past count are left
 * as they are). Keys use their low `bits` bits. *visible = count minus the
 * keys whose top digit of the reference's layout is all ones (16 bits: the
 * key; 24: its top 13 bits; 32: its top 16 bits). visible may be NULL.
 */
int rdx_sort(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits,
             uint32_t* ordering, uint64_t ordering_len, uint32_t* visible);

/*
 * WgpuRadixSort.sort (src/wgpu/WgpuRadixSort.ts:118-128): sort the first
 * `count` keys and values in place, ascending and stable; keys below 2^bits.
 * The result is always in the caller's buffers (no buffer swap).
 */
int rdx_sort_pairs(rdx_ctx* ctx, uint32_t* keys, uint32_t* values, uint64_t count, int bits);

/*
 * WgpuRadixSort.sortIndirect (WgpuRadixSort.ts:132-141): sort the first
 * min(*count_dev, capacity) pairs, with the count read on the device (device
 * pointers only; nothing is read back).
 */
int rdx_sort_pairs_indirect(rdx_ctx* ctx, uint32_t* keys, uint32_t* values,
                            const uint32_t* count_dev, uint64_t capacity, int bits);

/*
 * WgpuCompact.compact (src/wgpu/WgpuCompact.ts:22-132): the keys of the first
 * n that are not `invalid`, with their indices as values, to the front of
 * keys_out / values_out in input order; their number to *count_out.
 */
int rdx_compact(rdx_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t invalid,
                uint32_t* keys_out, uint32_t* values_out, uint32_t* count_out);

/*
 * WgpuSplatSorter.sort (src/wgpu/WgpuSplatSorter.ts:64-71): compact away the
 * invalid keys (2^bits - 1) of `count` projected keys, sort the rest back to
 * front: values[i] is the i-th splat drawn, *count_out the visible count, and
 * draw_args (5 x uint32, may be NULL) the drawIndexedIndirect arguments
 * [6 * 1024, ceil(visible / 1024), 0, 0, 0] (WgpuSplatSorter.ts:46-57).
 */
int rdx_splat_sort(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits,
                   uint32_t* values, uint32_t* count_out, uint32_t* draw_args);

/* ---- projection ---- */

/*
 * projectCollection (src/render/SplatProjector.ts:106-139) with the ewa
 * method: every object's splats through its SH (from the head, in object
 * space), its transform to head space, and each eye's EWA projection, fused
 * in one launch. pass RDX_PASS_KEYS writes keys only. cull_keys: keys of
 * splats culled in every eye are invalid (the GPU sort's order); else only
 * invisible splats and those outside params.sort_guard get it.
 */
int rdx_project(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                const rdx_params* params, int sort_bits, int pass, int cull_keys,
                const rdx_outputs* out);

/*
 * One frame: rdx_project (full pass, cull_keys on) then the stable sort of its
 * keys, as SplatRenderer.update runs it (SplatRenderer.ts:412-456):
 * ordering[i] (i < n) is the i-th splat back to front, culled splats last in
 * index order; *visible the number drawn. out->keys may be NULL (the keys then
 * live in scratch).
 */
int rdx_frame(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
              const rdx_params* params, int sort_bits, const rdx_outputs* out,
              uint32_t* ordering, uint32_t* visible);

/* ---- the projection methods ---- */

/*
 * ProjectionMethod (src/render/projections.tsl.ts:42, 469-474). ewa is the
 * method of rdx_project; the ray methods bound each splat per eye and keep its
 * 3D shape for the draw's ray evaluation:
 *   3dgut  a 2D bound from 7 sigma points (gutBound, projections.tsl.ts:183-220)
 *   htgs   the exact outline of the ellipsoid (htgsBound, 223-262)
 *   raygs  a tilted 3D quad facing the eye (raygsFrame / raygs, 336-467)
 */
#define RDX_METHOD_EWA 0
#define RDX_METHOD_3DGUT 1
#define RDX_METHOD_HTGS 2
#define RDX_METHOD_RAYGS 3

/* Words per splat of `method` with `eyes` eyes (ProjectionDef.headWords +
   eyes * eyeWords): 4E (ewa), 6 + 2E (3dgut, htgs), 4 + 3E (raygs); -1 when
   either is out of range. */
int rdx_method_words(int method, int eyes);

/*
 * The words and keys of one projection with `method`, as SplatProjection.write
 * stores them (src/render/SplatProjection.ts:139-153) for
 * projectCollection (SplatProjector.ts:106-139):
 *   words  uint32 [n][rdx_method_words(method, E)]: the head words, then each
 *          eye's, in the reference's order (projections.tsl.ts:5-17); the
 *          reference's channel c (w<c>, a uint32x4 or uint32x2 texture) holds
 *          words 4c .. 4c + 3 of a row. A culled eye's words are zero; the
 *          head words are zero when the head basis drops the splat (invisible,
 *          or its blur-compensated opacity below min_alpha).
 *   keys   uint32 [n], as rdx_project's (cull_keys: keys of splats that no
 *          eye shows are invalid).
 * Either output may be NULL. ewa forwards to rdx_project (its words output).
 * The ray methods take device memory only. Objects whose object-to-head
 * transform is a rotation times a uniform scale use transformUniform
 * (splatTransform.tsl.ts:143-152); other transforms and cov tables reach the
 * splat form through the covariance and fromCov (src/gpu/splats.tsl.ts:
 * 189-199), as the reference's transformSplat and transformForm do.
 */
int rdx_project_words(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                      const rdx_params* params, int method, int sort_bits, int cull_keys, uint32_t* words,
                      uint32_t* keys);

/* ---- the projection's gradient ---- */

/* Upstream gradients, laid out as rdx_project's outputs (float32, device
   memory; NULL: zero), and the forward's opacity output, which says which
   eyes drew each splat (nonzero: drawn). */
typedef struct rdx_grads_in {
  const float* mean2d;      /* [E][n][2]: dL/d(mean2d), pixels */
  const float* conic;       /* [E][n][3] */
  const float* depth;       /* [E][n] */
  const float* opacity;     /* [E][n] */
  const float* rgb;         /* [E][n][3] */
  const float* fwd_opacity; /* [E][n], required */
} rdx_grads_in;

/* One object's gradient rows, float32 device memory in the table's shapes
   (rows [0, count) are written; NULL: not wanted). */
typedef struct rdx_table_grads {
  float* centers;     /* [count][3] */
  float* log_scales;  /* [count][3] */
  float* quats;       /* [count][4]: of the stored, unnormalised quaternion */
  float* opacities;   /* [count] */
  float* colors;      /* [count][1 + K][3]: base rgb, then the SH coefficients (float32 also for float16 tables) */
} rdx_table_grads;

/*
 * The gradient of rdx_project's full pass (mean2d, conic, depth, opacity,
 * rgb) with respect to raw tables' fields, computed in float64 by one thread
 * per splat; grads[k] receives object k's rows. Same objects, camera and
 * params as the forward. An eye that culled a splat contributes nothing; the
 * rgb clamp (max(base + SH, 0)) passes a gradient only where it is open.
 * RDX_ERR_UNSUPPORTED for ext tables (quantised words have no gradient).
 * No counterpart in the reference, which renders only.
 */
int rdx_project_backward(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                         const rdx_params* params, const rdx_grads_in* upstream, const rdx_table_grads* grads);

/* ---- PLY files to raw tables ---- */

/* What a PLY file holds (its header): splats, SH degree (from its f_rest_*
   properties, ply.ts shDegree) and kind: 0 standard 3DGS, 1 RGB point
   cloud, 2 SuperSplat / PlayCanvas compressed */
typedef struct rdx_ply_info {
  uint64_t count;
  int32_t sh_degree;
  int32_t kind;
} rdx_ply_info;
int rdx_ply_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_ply_info* info);

/*
 * PlyFile.read (src/core/ply.ts:58-264) of a binary PLY file (host or device
 * bytes) into the columns of a raw table with `count` rows: centers [3],
 * log_scales [3], quats [4] (normalised x y z w; 16-byte aligned), opacities,
 * colors [1 + K][3] (base rgb = 0.5 + SH_C0 f_dc, then the SH coefficients
 * coefficient-major) of degree sh_degree (-1: the file's; at most the file's).
 * Any output may be NULL. Errors carry the reference's texts ("PLY has no
 * vertex element", "PLY vertex lacks ...", "PLY file ended unexpectedly" ...).
 */
int rdx_decode_ply(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, int sh_degree, float* centers,
                   float* log_scales, float* quats, float* opacities, float* colors);

/* ---- SPZ files to raw tables ---- */

/* What an SPZ file holds (its header; unpackSpz, src/core/spz.ts:141-263):
   splats, version (1-4), SH degree (0-4), fractional bits of its fixed-point
   centres, flags, and container: 0 gzip (versions 1-4), 1 SPZ 4's NGSP
   container (zstd streams). */
typedef struct rdx_spz_info {
  uint64_t count;
  int32_t version;
  int32_t sh_degree;
  int32_t fractional_bits;
  int32_t flags;
  int32_t container;
  int32_t reserved;
} rdx_spz_info;
int rdx_spz_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_spz_info* info);

/*
 * SpzFile.read (src/core/spz.ts:265-348) of an SPZ file in HOST memory (the
 * container is unpacked on the host: zlib for gzip, libzstd for SPZ 4) into the
 * columns of a raw table with `count` rows, decoded on the device: centers [3],
 * log_scales [3] (byte / 16 - 10), quats [4] (normalised x y z w; 16-byte
 * aligned), opacities (alpha / 255), colors [1 + K][3] (base rgb
 * (b / 255 - 0.5) SH_C0 / 0.15 + 0.5, then (b - 128) / 128 coefficient-major)
 * of degree sh_degree (-1: the file's; at most the file's). Any output may be
 * NULL. Trailers (LoD tree, PBR) and extension records are not decoded. Errors
 * carry the reference's texts ("Invalid SPZ file", "Unsupported SPZ version
 * ...", "SPZ 4 stream ... sizes don't match its header" ...).
 */
int rdx_decode_spz(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, int sh_degree, float* centers,
                   float* log_scales, float* quats, float* opacities, float* colors);

/* ---- RDX files (the reference's own container) to device arrays ---- */

/* What an RDX file holds (its header piece; src/core/rdx.ts:19-40, 162-170):
   elements, rows per chunk, chunks, serialized channels, and the header's JSON
   text (bundle definitions and metas) */
typedef struct rdx_rdxfile_info {
  uint64_t count;
  uint64_t chunk_size;
  int32_t n_chunks;
  int32_t n_channels;
  uint64_t header_json_bytes;
} rdx_rdxfile_info;
/* One serialized channel, in payload order: bundle and label names, its
   ArrayFormats name ("uint32x4", "float16", ...) and bytes per element */
typedef struct rdx_rdxfile_channel {
  char bundle[64];
  char label[64];
  char format[16];
  int32_t element_bytes;
  int32_t reserved;
} rdx_rdxfile_channel;
/* Fills info; then up to `capacity` channels and up to json_capacity bytes of
   the header's JSON (either may be NULL). Host bytes only. */
int rdx_rdxfile_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_rdxfile_info* info,
                          rdx_rdxfile_channel* channels, int capacity, char* header_json, uint64_t json_capacity);

/*
 * RdxFile.read of a whole file in HOST memory (header then every chunk;
 * decodeRdxChunk, src/core/rdx.ts:181-205): channels[k] (n_channels pointers,
 * host or device, NULL to skip) receives channel k's count * element_bytes
 * bytes. Payloads are inflated on the host and transposed back on the device.
 * Errors carry the reference's texts ("Not an RDX piece of the expected
 * type", "RDX version ... is not 1", "Chunk at ...: ... holds ... bytes,
 * expected ...").
 */
int rdx_decode_rdxfile(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, void* const* channels);

/* ---- batched frames: many views of many collections ---- */

/* One view of a batch: a collection (objects, as for rdx_frame) and its camera. */
typedef struct rdx_view {
  const rdx_object* objects;
  int n_objects;
  int reserved;
  const rdx_camera* camera;
} rdx_view;

/*
 * Several frames in one call: each view is the SplatRenderer.update of its own
 * collection and camera (SplatRenderer.ts:412-456), run as one projection
 * launch per table kind and one segmented sort with a segment per view. View
 * v's splats are output rows [first_v, first_v + n_v), first_v = n_0 + ... +
 * n_{v-1}, n_v its objects' counts summed; eye e of row r is output e * N + r
 * (N = all rows; every view has the same number of eyes). ordering[first_v + i]
 * is view v's i-th splat back to front, an index within the view; visible[v]
 * its drawn count (n_views words). The results equal n_views rdx_frame calls.
 */
int rdx_frame_batched(rdx_ctx* ctx, const rdx_view* views, int n_views, const rdx_params* params,
                      int sort_bits, const rdx_outputs* out, uint32_t* ordering, uint32_t* visible);

/*
 * A batched frame captured once in a CUDA graph and replayed: rdx_batch_create
 * plans it, allocates its scratch (descriptors, keys, sort state, lookback)
 * and captures its kernels; every rdx_batch_launch is one cudaGraphLaunch on
 * the context's stream. Tables, outputs, ordering and visible must be device
 * memory that stays valid while the batch exists. rdx_batch_update replaces
 * the cameras, object matrices and parameters (same views, tables and counts)
 * for the launches enqueued after it, without capturing again.
 * rdx_batch_synchronize waits for the stream and reports RDX_ERR_TIMEOUT if a
 * bounded device wait gave up. No counterpart in the reference: it dispatches
 * every object and view separately (SplatProjector.ts:106-139).
 */
typedef struct rdx_batch rdx_batch;
int rdx_batch_create(rdx_ctx* ctx, const rdx_view* views, int n_views, const rdx_params* params,
                     int sort_bits, const rdx_outputs* out, uint32_t* ordering, uint32_t* visible,
                     rdx_batch** batch);
int rdx_batch_update(rdx_batch* batch, const rdx_view* views, int n_views, const rdx_params* params);
int rdx_batch_launch(rdx_batch* batch);
int rdx_batch_synchronize(rdx_batch* batch);
int rdx_batch_launches(const rdx_batch* batch, uint64_t* launches);  /* kernels per launch */
int rdx_batch_destroy(rdx_batch* batch);

/*
 * Autotuning. rdx_batch_tune times, on the batch's own buffers and stream
 * (CUDA events, the median of `reps` frames after one warm-up each), the
 * projection at 2, 4 and 8 warps per block and then every digit-pass variant
 * the batch can take; it keeps the fastest pair (never slower than the
 * defaults, which are candidate 0), captures the batch's graph again with
 * it, and remembers it in the context for frames of the same shape (key
 * width, one view or many, the row count's power of two, the first table's
 * kind). rdx_sort_tune does the same for one-segment sorts of `count` device
 * keys (the keys are read, not changed). Both synchronise the stream.
 * No counterpart in the reference, whose keysPerThread is chosen by hand.
 */
#define RDX_TUNE_MAX 16
typedef struct rdx_tune_result {
  int32_t sort_variant;          /* chosen digit-pass variant */
  int32_t project_warps;         /* chosen warps per projection block (0: no projection) */
  int32_t candidates;            /* entries below */
  int32_t reserved;
  double default_ms;             /* a frame (sort) with the defaults */
  double tuned_ms;               /* with the choice */
  int32_t cand_sort[RDX_TUNE_MAX];
  int32_t cand_warps[RDX_TUNE_MAX];
  double cand_ms[RDX_TUNE_MAX];  /* median ms of each candidate */
} rdx_tune_result;
int rdx_batch_tune(rdx_batch* batch, int reps, rdx_tune_result* out);
int rdx_sort_tune(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits, int reps, rdx_tune_result* out);

/* ---- sorting without allocating ---- */

/*
 * SortKeys.sort for callers that may not allocate GPU memory: hosts that own
 * the whole device memory budget, or frame loops where an allocation's device
 * synchronisation would stall. Same order and visible count as rdx_sort, for
 * up to 2^20 keys (RDX_ERR_CAPACITY beyond), with scratch in a fixed device
 * array of the library (about 18 MB on every GPU that loads it, until exit)
 * instead of allocated memory; it allocates nothing and takes no context.
 * keys, ordering and visible (may be NULL) must be device memory
 * (RDX_ERR_ARG otherwise). The work is enqueued on `stream` (NULL: the legacy
 * default stream); *visible becomes 0xffffffff if a bounded device wait gave
 * up, and with visible == NULL such a wait goes unreported. Every call looks
 * up the array's device address on the current device (no cached address
 * outlives a context); the first call on a device also loads the library's
 * device code there, so make it before capturing a stream. All calls share
 * the array: calls that overlap on the GPU race; issue them one after another.
 * No counterpart in the reference: its sorts allocate their buffers.
 */
int rdx_sort_noalloc(const uint32_t* keys, uint64_t count, int bits, uint32_t* ordering,
                     uint64_t ordering_len, uint32_t* visible, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RADIX_B200_H */
