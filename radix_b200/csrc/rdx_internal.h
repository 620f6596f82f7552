// Internal declarations shared by the CUDA sources and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/radix_b200.h"

namespace rdx {

// ---- sort ----

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per onesweep tile
constexpr int kRadix = 256;
constexpr int kMaxPasses = 4;
// Lookback words: a 2-bit flag over a 30-bit count, so a segment holds < 2^30 keys
constexpr uint32_t kMaxSegmentKeys = (1u << 30) - 1u;
// Bounded device waits: polls of a lookback word before the kernel gives up
constexpr uint32_t kSpinLimit = 1u << 22;

// Segments of one sort, in device memory: seg_off[S + 1] element offsets,
// seg_tiles[S + 1] the running count of 4096-key tiles. A sort of one array
// is one segment.
struct SortSegments {
  const uint64_t* seg_off;
  const uint32_t* seg_tiles;
  int count;            // S
  uint32_t max_tiles;   // grid size: at least seg_tiles[S]
};

// Device scratch of a sort (all in one context allocation)
struct SortScratch {
  uint32_t* hist;        // [S][passes][256]
  uint32_t* ref_hidden;  // [S] keys the reference's visible count leaves out
  uint32_t* counters;    // [passes] tile counters
  uint32_t* lookback;    // [passes][max_tiles][256]
  uint32_t* keys_a;      // [n] ping-pong
  uint32_t* vals_a;
  uint32_t* keys_b;
  uint32_t* vals_b;
};

// Sort segments of keys_in (values: vals_in, or each key's index within its
// segment when vals_in is null) into keys_out / vals_out (keys_out may be null:
// values only). The result is stable and ascending by the low `bits` bits.
// Everything is enqueued on `stream`; error_flag (device) is set on a timeout.
cudaError_t sort_segments(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                          uint32_t* vals_out, const SortSegments& segs, int bits,
                          const SortScratch& scratch, uint32_t* error_flag, cudaStream_t stream);

// Bytes of memset-zeroed state at the head of the scratch (hist, ref_hidden, counters)
size_t sort_small_state_words(int segments, int passes);

// ---- keys, compaction ----

cudaError_t launch_keys_f64(const double* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s);
cudaError_t launch_keys_f32(const float* d, uint64_t n, int bits, uint32_t* keys, cudaStream_t s);
// visible[s] = seg_len - ref_hidden[s]
cudaError_t launch_visible(const uint64_t* seg_off, const uint32_t* ref_hidden, int segments,
                           uint32_t* visible, cudaStream_t s);
// Order-preserving compaction of keys != invalid; lookback: [tiles] zeroed here
cudaError_t launch_compact(const uint32_t* keys, uint64_t n, uint32_t invalid, uint32_t* keys_out,
                           uint32_t* vals_out, uint32_t* count_out, uint32_t* lookback,
                           uint32_t* error_flag, cudaStream_t s);
// seg_off = {0, min(*count, capacity)}, seg_tiles = {0, tiles}
cudaError_t launch_indirect_segments(const uint32_t* count, uint64_t capacity, uint64_t* seg_off,
                                     uint32_t* seg_tiles, cudaStream_t s);
cudaError_t launch_draw_args(const uint32_t* count, uint32_t* args, cudaStream_t s);

// ---- projection ----

struct DevTable {
  int layout;
  int sh_degree;
  int color_dtype;
  int reserved;
  const float* centers;
  const float* log_scales;
  const float* quats;
  const float* opacities;
  const void* colors;
  const uint32_t* ext_a;
  const uint32_t* ext_b;
  const uint32_t* ext_sh[6];
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
  uint32_t first_tile;   // running count of 256-splat tiles before this object
  uint32_t reserved2;
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
};

constexpr int kProjThreads = 256;

// One launch over every descriptor (a collection): descs in device memory
cudaError_t launch_project(const ProjDesc* descs_dev, const ProjDesc* descs_host, int n_desc,
                           uint32_t total_tiles, const ProjOutputs& out, cudaStream_t stream);

}  // namespace rdx
