// Internal declarations shared by the CUDA sources and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "../../include/radix_b200.h"

namespace rdx {

// ---- programmatic dependent launch ----
// A kernel launched with launch_after() may start while the kernel before it
// in the stream is still running, once every block of that kernel has called
// pdl_trigger() (or exited); it calls pdl_wait() before it touches anything
// the earlier kernel writes, which returns when that kernel has completed and
// its writes are visible. Both are no-ops in a kernel launched plainly, and
// the launch attribute has no effect when the previous operation in the
// stream is not a kernel (a copy or a memset keeps full ordering).
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... Params, typename... Args>
cudaError_t launch_after(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                         Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif

// ---- the device error flag ----
// Bits of a context's (or batch's) device error word: a bounded wait gave
// up; an index a kernel computed fell outside its buffer (the kernels clamp
// such accesses; a build with RDX_CHECK defined also records that they did,
// since a correct launch never clamps)
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrBounds = 2u;
#ifdef __CUDACC__
__device__ __forceinline__ void check_failed(uint32_t* flag) {
#ifdef RDX_CHECK
  if (flag) atomicOr(flag, kErrBounds);
#else
  (void)flag;
#endif
}
#endif

// ---- sort ----

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per onesweep tile
// Sorts of at most kSmallSortTiles such tiles run their digit passes in tiles of
// kSortThreads * kSmallItems keys (when their lookback words allow)
constexpr int kSmallItems = 4;
constexpr uint32_t kSmallSortTiles = 256;
constexpr int kRadix = 256;
constexpr int kMaxPasses = 4;
// Lookback words: a 2-bit flag over a 30-bit count, so a segment holds < 2^30 keys
constexpr uint32_t kMaxSegmentKeys = (1u << 30) - 1u;
// Bounded device waits: polls of a lookback word before the kernel gives up
constexpr uint32_t kSpinLimit = 1u << 22;
// Digit passes of a one-segment sort in one cooperative kernel (SortCall.coop):
// threads per block x keys per thread of a sub-tile
constexpr int kCoopNone = 0;
constexpr int kCoop1024x16 = 1;
constexpr int kCoop512x16 = 2;
constexpr int kCoop1024x8 = 3;
constexpr int kCoopVariants = 4;
// Blocks a cooperative sort may have (2 per SM on up to 256 SMs): its per-block counts
constexpr uint32_t kMaxCoopBlocks = 512;

// Segments of one sort, in device memory: segment s is [begin[s], end[s]);
// tiles[S + 1] is the running count of 4096-key tiles. A sort of one array is
// one segment.
struct SortSegments {
  const uint64_t* begin;
  const uint64_t* end;
  const uint32_t* tiles;
  int count;            // S
  uint32_t max_tiles;   // grid size: at least tiles[S]
};

// Device scratch of a sort (carved from a context's arena)
struct SortScratch {
  uint32_t* hist;        // [S][passes][256] digit counts of the valid keys
  uint32_t* valid;       // [S] keys below 2^bits - 1
  uint32_t* ref_hidden;  // [S] keys the reference's visible count leaves out
  uint32_t* counters;    // [passes + 1] tile counters (the last: the partition's)
  uint32_t* tile_valid;  // [max_tiles] valid keys of each tile
  uint64_t* vbegin;      // [S] segments of the valid keys (passes after the first)
  uint64_t* vend;        // [S]
  uint32_t* vtiles;      // [S + 1]
  uint32_t* keys_a;      // [n] ping-pong
  uint32_t* vals_a;
  uint32_t* keys_b;
  uint32_t* vals_b;
  uint32_t* block_counts;  // [kMaxCoopBlocks][256] of a cooperative sort (null: none)
};

// hist, valid, ref_hidden, counters and tile_valid are contiguous: words zeroed before a sort
size_t sort_small_state_words(int segments, int passes, uint32_t max_tiles);
// The digit passes' tile count of a small sort (0: not small); lookback words
// for passes * max(this, max_tiles) * kRadix let a sort use small tiles
uint32_t sort_small_pass_tiles(uint32_t max_tiles);

// Sort segments of keys_in (values: vals_in, or each key's index within its
// segment when vals_in is null) into keys_out / vals_out (keys_out may be null:
// values only), stable and ascending by the low `bits` bits; the largest key
// 2^bits - 1 goes to each segment's tail in input order. zeroed: the caller
// has zeroed the small state (sort_small_state_words from scratch.hist), so
// the sort starts with a kernel; else it zeroes it first. The lookback
// words [passes][max_tiles][256] are tagged with the epoch in the device word
// `epoch`, which the sort advances on the device before its first pass (zero
// it with the lookback words; it needs no host update between calls).
struct SortCall {
  const uint32_t* keys_in;
  const uint32_t* vals_in;
  uint32_t* keys_out;
  uint32_t* vals_out;
  SortSegments segs;
  int bits;
  bool zeroed;      // the small state is zeroed already
  bool no_drop;     // rank the largest key like the others
  SortScratch scratch;
  uint64_t* lookback;
  uint64_t lookback_words;  // its capacity
  uint32_t* epoch;
  uint32_t* error_flag;
  uint32_t spin_limit = 0;  // polls of a bounded device wait (0: kSpinLimit)
  int silent_pass = -1;     // a digit pass whose first tile publishes no lookback word (a test hook; -1: none)
  int coop = kCoopNone;     // one segment: the digit passes in this cooperative variant (needs block_counts)
  int pass_items = 0;       // onesweep digit passes after a partition: keys a thread (4, 8, 16; 0: by size)
  // Per segment (may be null): the reference's visible count, (end - begin) - ref_hidden
  // (visible_ref), or the valid keys; the partition writes it, else a kernel after the passes
  uint32_t* visible = nullptr;
  bool visible_ref = false;
};
cudaError_t sort_segments(const SortCall& call, cudaStream_t stream, int* launches);
// Blocks of a cooperative variant resident on the current device (0: it cannot launch)
int coop_blocks(int variant);

// ---- keys, compaction ----

cudaError_t launch_keys_f64(const double* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s);
cudaError_t launch_keys_f32(const float* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s);
// visible[s] = (end - begin) - ref_hidden[s], or valid[s] (ref_hidden null)
cudaError_t launch_visible(const uint64_t* begin, const uint64_t* end, const uint32_t* ref_hidden,
                           const uint32_t* valid, int segments, uint32_t* visible, cudaStream_t s);
// Order-preserving compaction of keys != invalid (three launches); tile_valid:
// ceil(n / 4096) words of scratch
cudaError_t launch_compact(const uint32_t* keys, uint64_t n, uint32_t invalid, uint32_t* keys_out,
                           uint32_t* vals_out, uint32_t* count_out, uint32_t* tile_valid,
                           uint32_t* error_flag, cudaStream_t s);
// One segment [0, min(*count, capacity)) and its tiles
cudaError_t launch_indirect_segments(const uint32_t* count, uint64_t capacity, uint64_t* begin, uint64_t* end,
                                     uint32_t* tiles, cudaStream_t s);
cudaError_t launch_draw_args(const uint32_t* count, uint32_t* args, cudaStream_t s);

// ---- projection ----

struct DevTable {
  int layout;
  int sh_degree;
  int color_dtype;
  int sh_codec;
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
  const uint32_t* sh_palette;  // SH from a palette when set (entries of sh_stride texels)
  const uint16_t* sh_label;
  uint32_t sh_stride;
  uint32_t sh_palette_size;
};

struct DevParams {
  float max_std_dev, min_alpha, blur_amount, pre_blur_amount, clip_xy, min_pixel_radius,
      max_pixel_radius, min_contribution, focal_distance, aperture_tan, sort_guard;
  int lod_inflate;
  int max_sh_degree;
  int reserved;
};

struct DevEye {
  double from_head[12];  // rows of the 3x4 head -> eye transform
  double proj[16];       // column-major projection
  double wd[9];          // object -> eye 3x3, row-major (from_head3 * a3)
  double focal_d[2];     // size / 2 * (P00, P11)
  float proj11;          // projection element (1, 1) for the depth of field
  int identity;          // from_head is exactly the identity
  int ortho;
  int reserved;
};

// One object of a projection (one view of it): everything the kernel reads
struct ProjDesc {
  DevTable table;
  DevParams params;
  double a[12];          // rows of the 3x4 object -> head transform
  double origin[3];      // the head in object space (SH view origin)
  int degenerate;        // the object's 3x3 is zero: every splat is invisible
  uint64_t count;        // splats of the object
  uint64_t out_offset;   // output index of its first splat
  uint64_t out_n;        // outputs per eye (stride between eyes)
  DevEye eye[2];
  double width, height, ndc_z_min;
  int eyes;
  int sort_bits;
  int cull_keys;
  int keys_only;
  uint32_t first_tile;   // running count of projection tiles before this object
  int object;            // index of the object in its view's collection
  int segment;           // the sort segment the keys belong to (a view of a batch)
  uint32_t host_row_bytes;  // bytes a drawn candidate reads from host memory in place (0: none)
};

struct ProjOutputs {
  float* mean2d;
  float* conic;
  float* depth;
  float* opacity;
  float* rgb;
  float* radii;
  uint32_t* words;
  uint32_t* keys;
  // Words the launch's first block zeroes (the sort's small state, so that no
  // memset separates the projection from the sort's kernels); may be null
  uint32_t* zero;
  uint64_t zero_words;
  uint32_t* check_flag;  // the device error word (bounds-checked builds record clamped rows there)
  unsigned long long* host_bytes;  // adds host_row_bytes for each candidate of an object read in place (may be null)
};

// Splats per projection chunk (one warp)
constexpr int kProjTile = 32;


// ---- SPZ files (src/core/spz.ts) to raw tables ----

// An SPZ file's header and the layout of its byte columns once unpacked on the
// host: centers, alphas, colors, scales, rotations, SH, back to back
struct SpzDesc {
  uint64_t count = 0;
  int container = 0;  // 0: gzip (versions 1-4), 1: SPZ 4's NGSP container
  int version = 0;
  int sh_degree = 0;
  int fractional_bits = 0;
  int flags = 0;
  int out_degree = 0;
  int n_streams = 0;           // NGSP: zstd streams (non-empty columns)
  uint64_t toc_at = 0;         // NGSP: byte offset of the table of contents
  uint64_t col_off[6] = {};    // in the unpacked payload
  uint64_t col_size[6] = {};
  uint64_t payload = 0;        // unpacked bytes
  const unsigned char* base = nullptr;  // device address of the unpacked payload (set before a launch)
};
constexpr int kSpzGzip = 0;
constexpr int kSpzNgsp = 1;
// An SPZ file's header from host bytes: null, or the reference's error text
const char* spz_header(const unsigned char* bytes, uint64_t nbytes, SpzDesc* d);
// The file's columns unpacked on the host into payload (d.payload bytes): gzip
// inflated by zlib, NGSP streams by libzstd (loaded when first needed): null or an error text
const char* spz_unpack(const unsigned char* bytes, uint64_t nbytes, const SpzDesc& d, unsigned char* payload);
cudaError_t launch_decode_spz(const SpzDesc& d, float* centers, float* log_scales, float* quats, float* opacities,
                              float* colors, cudaStream_t stream);

// ---- RDX files (src/core/rdx.ts): serialized ArrayData bundles ----

struct RdxChannel {
  std::string bundle, label, format;
  int element_bytes;
};
struct RdxFile {
  uint64_t count = 0;
  uint64_t chunk_size = 0;
  uint64_t header_bytes = 0;  // where chunk 0 starts
  std::vector<RdxChannel> channels;   // payload order
  std::vector<uint64_t> chunk_bytes;
  std::string header_json;
};
// One chunk's channel inflated on the host: its transposed bytes at `src` of the staged buffer
struct RdxSpan {
  uint64_t src;
  int channel;
  uint64_t start;
  uint32_t count;
  uint32_t bytes;
};
// The same on the device: where its elements go
struct RdxPiece {
  uint64_t src;
  unsigned char* dst;
  uint32_t count;
  uint32_t bytes;
};
// fn(0) .. fn(n - 1) shared among host threads (a thread per MB of work_bytes
// at most, up to the host's threads), returning when all are done
void parallel_for(size_t n, uint64_t work_bytes, const std::function<void(size_t)>& fn);
// An RDX file's header from host bytes: null, or the reference's error text
const char* rdxfile_header(const unsigned char* bytes, uint64_t nbytes, RdxFile* f);
// Every chunk's payloads of the wanted channels inflated into `staged`: null or an error text
const char* rdxfile_unpack(const unsigned char* bytes, uint64_t nbytes, const RdxFile& f, const bool* wanted,
                           std::vector<unsigned char>* staged, std::vector<RdxSpan>* spans);
// The staged bytes transposed back into the pieces' destinations (one launch
// per 65535 pieces; pieces_host is the host copy of pieces_dev)
cudaError_t launch_untranspose(const RdxPiece* pieces_dev, const RdxPiece* pieces_host, int n_pieces,
                               const unsigned char* staged, cudaStream_t stream);

// One persistent launch over every descriptor of one table kind (descs in device memory)
// ---- PLY files (src/core/ply.ts) to raw tables ----

constexpr int kPlyRest = 72;  // f_rest_* values of SH degree 4

// A scalar property of a record: byte offset (-1: absent) and type
// (0 char, 1 uchar, 2 short, 3 ushort, 4 int, 5 uint, 6 float, 7 double)
struct PlyProp {
  int32_t offset;
  int32_t type;
};

enum PlyKind { kPlyStandard = 0, kPlyPoints = 1, kPlyCompressed = 2 };

// Where a file's values are, with the header already read on the host
struct PlyDesc {
  int32_t kind;
  int32_t little;           // binary_little_endian
  int32_t sh_degree;        // of the file
  int32_t out_degree;       // of the rows written
  uint64_t count;           // splats
  const unsigned char* vertex;  // the first vertex record (device memory)
  uint32_t record;          // bytes per vertex record
  PlyProp xyz[3], scale[3], rot[4], opacity, color[3], alpha;
  PlyProp rest[kPlyRest];   // coefficient-major (value 3k + c is f_rest_{c * N + k})
  // compressed files: per-chunk ranges and packed words
  const unsigned char* chunk;
  uint32_t chunk_record;
  PlyProp chunk_prop[18];   // min/max x y z, min/max scale x y z, min/max r g b (absent: 0, 0, 0, 1, 1, 1)
  PlyProp packed[4];        // packed_position, packed_rotation, packed_scale, packed_color
  const unsigned char* sh;  // the sh element (null: none)
  uint32_t sh_record;
  int32_t sh_byte[kPlyRest]; // coefficient-major byte offsets in an sh record
};

// Host: read a PLY header (the first bytes of a file of nbytes) into desc;
// 0 or an error text. vertex, chunk and sh are byte offsets into the file.
const char* parse_ply_header(const unsigned char* head, uint64_t head_bytes, uint64_t nbytes, PlyDesc* desc);

// Device: rows [0, count) of a raw table of degree out_degree
cudaError_t launch_decode_ply(const PlyDesc& desc, float* centers, float* log_scales, float* quats, float* opacities,
                              float* colors, cudaStream_t stream);

// ---- the projection's gradient (raw tables) ----

// Upstream gradients laid out as the forward's outputs ([E][n]...; null: zero)
// and the forward's opacity output, which marks the eyes that drew a splat
struct GradsIn {
  const float* mean2d;
  const float* conic;
  const float* depth;
  const float* opacity;
  const float* rgb;
  const float* fwd_opacity;
};

// One object's gradient rows (float32, the table's shapes; null: not wanted)
struct GradsOut {
  float* centers;
  float* log_scales;
  float* quats;
  float* opacities;
  float* colors;
};

// grads_dev[k] belongs to descs_dev[k]; one launch per table kind
cudaError_t launch_project_backward(const ProjDesc* descs_dev, const GradsOut* grads_dev, const ProjDesc* descs_host,
                                    int n_desc, uint32_t total_chunks, const GradsIn& in, cudaStream_t stream);

// warps: warps per block (2, 4 or 8; 0: 4)
cudaError_t launch_project(const ProjDesc* descs_dev, const ProjDesc* descs_host, int n_desc,
                           uint32_t total_tiles, const ProjOutputs& out,
                           uint32_t* error_flag, cudaStream_t stream, int warps = 0);
int project_warps_supported(int warps);
// Raw tables whose colour rows the projection may read from pinned host memory
// in place (a kernel flavour stages them a warp at a time)
bool project_host_rows_supported(const DevTable& t);

// ---- the ray projection methods (src/render/projections.tsl.ts:170-474) ----

constexpr int kMethodEwa = 0, kMethod3dgut = 1, kMethodHtgs = 2, kMethodRaygs = 3;

// What a ray method reads beside an object's ProjDesc: whether the object ->
// head transform is a rotation times a uniform scale, and then that rotation
// and scale (setTransform, src/render/splatTransform.tsl.ts:64-74; other
// transforms go through the covariance), and each eye's rotation from the
// head (SplatCamera.setViews, src/render/splatCamera.ts:129-131)
struct RayDesc {
  double tq[4];
  double tscale;
  double eye_q[2][4];
  int uniform;
  int reserved;
};

// rays_dev[k] belongs to descs_dev[k]; one launch per table kind; words
// [n][H + E * W] and keys [n] by each descriptor's out_offset
cudaError_t launch_project_rays(const ProjDesc* descs_dev, const RayDesc* rays_dev, const ProjDesc* descs_host,
                                int n_desc, uint32_t total_tiles, int method, uint32_t* words, uint32_t* keys,
                                cudaStream_t stream);

}  // namespace rdx
