// The C ABI (include/radix_b200.h): contexts, argument checks with the
// reference's error texts, staging of host buffers, the per-object and
// per-eye set-up of a camera in float64 (SplatCamera.setViews and
// setTransforms), and dispatch of the kernels on the context's stream.
//
// Host float64 maths here must round exactly as the oracle's: keep every sum
// in the same order and build with -ffp-contract=off.
#include <cuda_runtime.h>
#include <math.h>
#include <nvtx3/nvToolsExt.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <memory>
#include <new>
#include <vector>

#include "../../include/radix_b200.h"
#include "rdx_internal.h"

struct rdx_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string last_error;
  uint32_t* error_flag = nullptr;       // device word set by a bounded wait that gave up
  uint32_t* error_host = nullptr;       // pinned copy of it
  char* arena = nullptr;                // per-call device scratch
  size_t arena_bytes = 0;
  uint64_t launches = 0;                // kernels launched
  bool profiling = false;
  std::vector<cudaEvent_t> event_pool;  // free events
  struct Pending {
    int phase;
    cudaEvent_t start, stop;
  };
  std::vector<Pending> pending;         // recorded, not yet read
  double phase_ms[RDX_PHASES] = {0};
  uint64_t phase_runs[RDX_PHASES] = {0};
  // Pinned ring for small uploads (descriptors, segments): a copy from it is
  // asynchronous; before the ring wraps, the last copy issued from it is awaited
  char* ring = nullptr;
  size_t ring_off = 0;
  cudaEvent_t ring_event = nullptr;
  bool ring_used = false;
  // Lookback words of the onesweep passes, tagged with a per-sort epoch so
  // they never need clearing; zeroed once when (re)allocated. The epoch is a
  // device word (error_flag + 1) that each sort advances on the device.
  uint64_t* lookback = nullptr;
  size_t lookback_words = 0;
  // Bounded device waits: polls before a wait gives up (0: the default), and
  // the one-shot test hook that silences a digit pass's first tile
  uint32_t spin_limit = 0;
  int silent_pass = -1;
  // How sorts run their digit passes (rdx_ctx_set_sort_variant; -1: tuned or default)
  int sort_variant = -1;
  // Choices of rdx_batch_tune / rdx_sort_tune, by workload shape (tune_key)
  struct Tuned {
    int sort_variant;
    int project_warps;
  };
  std::map<uint64_t, Tuned> tuned;
  // Host tables (rdx_ctx_set_host_reads): read the drawn rows of pinned columns
  // in place, or copy every host column in; bytes moved since the last query
  int host_reads = RDX_HOST_IN_PLACE;
  unsigned long long* host_bytes_dev = nullptr;  // rows read in place (the projection counts them)
  uint64_t host_bytes = 0;                       // columns copied in
};

static const size_t kRingBytes = 4u << 20;

namespace {

int fail(rdx_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->last_error = buf;
  return code;
}

int cuda_fail(rdx_ctx* ctx, cudaError_t err, const char* what) {
  return fail(ctx, RDX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
}

#define RDX_CUDA(call, what)                       \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
  } while (0)

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool aligned(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

// The device address of pinned host memory mapped into `device`'s address
// space (null: not such memory, or memory pinned for another device, which is
// then copied instead of read in place)
const void* mapped_host(const void* p, int device) {
  if (!p) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost && a.device == device ? a.devicePointer : nullptr;
}

// Bump allocation over the context's arena: a dry run sizes it, the real run carves it
struct Arena {
  char* base;
  size_t used = 0;
  explicit Arena(char* b) : base(b) {}
  template <class T>
  T* take(size_t count) {
    used = (used + 255) & ~(size_t)255;
    T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
    used += count * sizeof(T);
    return p;
  }
};

int ensure_arena(rdx_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->arena_bytes) return RDX_OK;
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  if (ctx->arena) cudaFree(ctx->arena);
  ctx->arena = nullptr;
  ctx->arena_bytes = 0;
  size_t want = bytes + bytes / 4 + (1 << 20);
  if (cudaMalloc(&ctx->arena, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RDX_ERR_NOMEM, "could not allocate %zu bytes of device scratch", want);
  }
  ctx->arena_bytes = want;
  return RDX_OK;
}

// The status of a device error word's bits (cleared by the caller): a
// bounded wait that gave up, else a clamped index (bounds-checked builds)
int device_error(rdx_ctx* ctx, uint32_t bits) {
  if (bits & rdx::kErrTimeout) return fail(ctx, RDX_ERR_TIMEOUT, "a device wait gave up (lookback of a tile never published)");
  return fail(ctx, RDX_ERR_CUDA, "a device bounds check failed: a kernel computed an index outside its buffer");
}

// Wait for the stream and report a device-side error
int finish(rdx_ctx* ctx) {
  RDX_CUDA(cudaMemcpyAsync(ctx->error_host, ctx->error_flag, 4, cudaMemcpyDeviceToHost, ctx->stream), "error flag");
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  if (*ctx->error_host) {
    const uint32_t bits = *ctx->error_host;
    *ctx->error_host = 0;
    cudaMemsetAsync(ctx->error_flag, 0, 4, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return device_error(ctx, bits);
  }
  return RDX_OK;
}

// A phase between begin and end is timed with events on the stream when
// profiling, and marked on the host timeline as an NVTX range named like the
// reference's renderer phases ("project", "sort"; SplatRenderer.ts:141-142),
// which a profiler attached to the process shows (a no-op without one)
struct Phase {
  rdx_ctx* ctx;
  int phase;
  cudaEvent_t start = nullptr;
  bool marked = false;
  Phase(rdx_ctx* c, int p) : ctx(c), phase(p) {
    static const char* const kNames[RDX_PHASES] = {"project", "sort", "copy in", "copy out", "batch"};
    nvtxRangePushA(p >= 0 && p < RDX_PHASES ? kNames[p] : "radix_b200");
    marked = true;
    if (!ctx || !ctx->profiling) return;
    start = take_event(ctx);
    if (start) cudaEventRecord(start, ctx->stream);
  }
  void end() {
    if (marked) {
      nvtxRangePop();
      marked = false;
    }
    if (!start) return;
    cudaEvent_t stop = take_event(ctx);
    if (!stop) return;
    cudaEventRecord(stop, ctx->stream);
    ctx->pending.push_back({phase, start, stop});
    start = nullptr;
  }
  ~Phase() { end(); }
  static cudaEvent_t take_event(rdx_ctx* ctx) {
    if (!ctx->event_pool.empty()) {
      cudaEvent_t e = ctx->event_pool.back();
      ctx->event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return e;
  }
};

// Copy `bytes` of host memory to the device asynchronously through the ring
int upload(rdx_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return RDX_OK;
  const size_t need = (bytes + 255) & ~(size_t)255;
  if (need > kRingBytes) {  // too big for the ring: a pageable copy (synchronous staging)
    RDX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload");
    return RDX_OK;
  }
  if (ctx->ring_off + need > kRingBytes) {
    if (ctx->ring_used) RDX_CUDA(cudaEventSynchronize(ctx->ring_event), "ring wait");
    ctx->ring_off = 0;
  }
  char* slot = ctx->ring + ctx->ring_off;
  memcpy(slot, src, bytes);
  RDX_CUDA(cudaMemcpyAsync(dst, slot, bytes, cudaMemcpyHostToDevice, ctx->stream), "upload");
  RDX_CUDA(cudaEventRecord(ctx->ring_event, ctx->stream), "ring event");
  ctx->ring_used = true;
  ctx->ring_off += need;
  return RDX_OK;
}

bool valid_bits(int bits) { return bits == 16 || bits == 24 || bits == 32; }

uint32_t tiles_of(uint64_t n) { return (uint32_t)((n + rdx::kSortTile - 1) / rdx::kSortTile); }

// Lookback tiles a pass of a sort of max_tiles 4096-key tiles may use: room
// for 2048-key digit-pass tiles always, and 1024-key tiles for small sorts
size_t lookback_tiles(uint32_t max_tiles) {
  return std::max((size_t)max_tiles * 2, (size_t)rdx::sort_small_pass_tiles(max_tiles));
}

// Sort scratch for `segments` segments of `total` keys
rdx::SortScratch take_sort_scratch(Arena& a, int segments, int passes, uint64_t total) {
  rdx::SortScratch s{};
  // hist, valid, ref_hidden, counters and tile_valid contiguous (one memset); each
  // segment adds at most one partial tile
  const uint32_t max_tiles = tiles_of(total) + (uint32_t)segments;
  uint32_t* small = a.take<uint32_t>(rdx::sort_small_state_words(segments, passes, max_tiles));
  if (small) {
    s.hist = small;
    s.valid = small + (size_t)segments * passes * rdx::kRadix;
    s.ref_hidden = s.valid + segments;
    s.counters = s.ref_hidden + segments;
    s.tile_valid = s.counters + passes + 1;
  }
  s.vbegin = a.take<uint64_t>(segments);
  s.vend = a.take<uint64_t>(segments);
  s.vtiles = a.take<uint32_t>(segments + 1);
  // Ping-pong pairs: the partition and every pass but the last write one of them
  s.keys_a = a.take<uint32_t>(total);
  s.vals_a = a.take<uint32_t>(total);
  s.keys_b = a.take<uint32_t>(total);
  s.vals_b = a.take<uint32_t>(total);
  s.block_counts = segments == 1 ? a.take<uint32_t>((size_t)rdx::kMaxCoopBlocks * rdx::kRadix) : nullptr;
  return s;
}

// Segment descriptors in the arena
struct SegBufs {
  uint64_t* begin;
  uint64_t* end;
  uint32_t* tiles;
};

SegBufs take_segs(Arena& a, int segments) {
  SegBufs b;
  b.begin = a.take<uint64_t>(segments);
  b.end = a.take<uint64_t>(segments);
  b.tiles = a.take<uint32_t>(segments + 1);
  return b;
}

// Grow the context's lookback words to `words` (zeroed: epoch 0 is never used)
int ensure_lookback(rdx_ctx* ctx, size_t words) {
  if (words <= ctx->lookback_words) return RDX_OK;
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  if (ctx->lookback) cudaFree(ctx->lookback);
  ctx->lookback = nullptr;
  ctx->lookback_words = 0;
  const size_t want = words + words / 4 + 4096;
  if (cudaMalloc(&ctx->lookback, want * 8) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, RDX_ERR_NOMEM, "could not allocate %zu lookback words", want);
  }
  RDX_CUDA(cudaMemsetAsync(ctx->lookback, 0, want * 8, ctx->stream), "lookback clear");
  ctx->lookback_words = want;
  return RDX_OK;
}

// ---- float64 matrices, column-major (the same sums, in the same order, as the oracle) ----

void mat4_mul(const double a[16], const double b[16], double out[16]) {
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

int mat4_invert(const double m[16], double out[16]) {
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

const int kShCoeffs[5] = {0, 3, 8, 15, 24};

// ---- tables: checks and staging ----

// SH texels per entry of a codec and degree (src/core/sh.ts:13-24)
int sh_texels(int codec, int degree) {
  static const int kPackedTexels[5] = {0, 1, 2, 3, 5};
  if (degree <= 0) return 0;
  return codec == RDX_SH_PACKED ? kPackedTexels[degree] : (kShCoeffs[degree] + 3) / 4;
}

struct TableBytes {
  size_t centers, scales, quats, opacities, colors, words, sh_texels;
};

TableBytes table_bytes(const rdx_table& t, uint64_t n) {
  TableBytes b{};
  const int k = kShCoeffs[t.sh_degree];
  if (t.layout == RDX_LAYOUT_RAW) {
    b.centers = n * 12;
    b.scales = n * 12;
    b.quats = n * 16;
    b.opacities = n * 4;
    b.colors = n * (size_t)(1 + k) * 3 * (t.color_dtype == RDX_DTYPE_F16 ? 2 : 4);
  } else {
    b.words = n * 16;  // one uint32x4 per splat and column
    b.sh_texels = (size_t)sh_texels(t.sh_codec, t.sh_degree);
  }
  return b;
}

size_t color_vec_bytes(const rdx_table& t) {
  const int k = kShCoeffs[t.sh_degree];
  const size_t row = (size_t)(1 + k) * 3 * (t.color_dtype == RDX_DTYPE_F16 ? 2 : 4);
  return row % 16 == 0 ? 16 : (row % 8 == 0 ? 8 : (row % 4 == 0 ? 4 : 2));
}

const char* layout_name(int layout) {
  switch (layout) {
    case RDX_LAYOUT_EXT: return "ext";
    case RDX_LAYOUT_PACKED: return "packed";
    case RDX_LAYOUT_COV: return "cov";
    default: return "raw";
  }
}

int check_table(rdx_ctx* ctx, const rdx_table* t, int index) {
  if (!t) return fail(ctx, RDX_ERR_ARG, "object %d has no table", index);
  if (t->layout < RDX_LAYOUT_RAW || t->layout > RDX_LAYOUT_COV)
    return fail(ctx, RDX_ERR_UNSUPPORTED, "table layout %d (raw 0, ext 1, packed 2, cov 3)", t->layout);
  if (t->sh_degree < 0 || t->sh_degree > 4) return fail(ctx, RDX_ERR_ARG, "sh_degree %d (0 to 4)", t->sh_degree);
  if (t->layout == RDX_LAYOUT_RAW) {
    if (t->color_dtype != RDX_DTYPE_F32 && t->color_dtype != RDX_DTYPE_F16)
      return fail(ctx, RDX_ERR_ARG, "color_dtype %d", t->color_dtype);
    if (!t->centers || !t->log_scales || !t->quats || !t->opacities || !t->colors)
      return fail(ctx, RDX_ERR_ARG, "raw table of object %d: a column is NULL", index);
    return RDX_OK;
  }
  const char* name = layout_name(t->layout);
  if (t->layout == RDX_LAYOUT_PACKED) {
    if (!t->packed) return fail(ctx, RDX_ERR_ARG, "packed table of object %d: the packed column is NULL", index);
    if (!(t->packed_encoding[1] > t->packed_encoding[0]) || !(t->packed_encoding[3] > t->packed_encoding[2]))
      return fail(ctx, RDX_ERR_ARG, "packed table of object %d: encoding ranges are empty", index);
  } else if (!t->ext_a || !t->ext_b) {
    return fail(ctx, RDX_ERR_ARG, "%s table of object %d: word column A or B is NULL", name, index);
  }
  if (t->sh_codec != RDX_SH_EXT && t->sh_codec != RDX_SH_PACKED)
    return fail(ctx, RDX_ERR_ARG, "%s table of object %d: SH codec %d (ext 0, packed 1)", name, index, t->sh_codec);
  const int texels = sh_texels(t->sh_codec, t->sh_degree);
  if (t->sh_palette) {
    if (!t->sh_label) return fail(ctx, RDX_ERR_ARG, "%s table of object %d: a palette without labels", name, index);
    if (t->sh_palette_size == 0 || t->sh_stride < (uint32_t)texels)
      return fail(ctx, RDX_ERR_ARG, "%s table of object %d: palette stride %u below the codec's %d texels", name, index,
                  t->sh_stride, texels);
  } else {
    for (int c = 0; c < texels; c++)
      if (!t->ext_sh[c]) return fail(ctx, RDX_ERR_ARG, "%s table of object %d: SH texel channel %d is NULL", name, index, c);
  }
  return RDX_OK;
}

// A column as the kernels read it: the caller's device pointer, pinned host
// memory in place (`in_place`: a column that only drawn candidates read, whose
// rows then cross the bus alone; *row_bytes grows by the bytes of its row), or
// a staged copy of host memory
template <class T>
const T* stage_column(rdx_ctx* ctx, Arena& a, const T* src, size_t bytes, size_t align, int* status,
                      bool in_place = false, uint64_t n = 0, uint32_t* row_bytes = nullptr) {
  if (is_device_ptr(src)) {
    if (!aligned(src, align)) *status = fail(ctx, RDX_ERR_ARG, "a device column is not %zu-byte aligned", align);
    a.take<char>(0);
    return src;
  }
  if (in_place && ctx->host_reads == RDX_HOST_IN_PLACE && n > 0) {
    const void* m = mapped_host(src, ctx->device);
    if (m && aligned(m, align)) {
      if (row_bytes) *row_bytes += (uint32_t)(bytes / n);
      a.take<char>(0);
      return reinterpret_cast<const T*>(m);
    }
  }
  char* dst = a.take<char>(bytes);
  if (dst && bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) *status = cuda_fail(ctx, e, "copy of a host column");
    ctx->host_bytes += bytes;
  }
  return reinterpret_cast<const T*>(dst);
}

// A table whose columns the kernels can read: the caller's device pointers,
// staged copies of host columns, and (pinned host memory, `in_place`) a raw
// SH-3 table's colour rows, which only drawn candidates read, in place;
// *row_bytes: the bytes of a candidate's row read in place
rdx::DevTable stage_table(rdx_ctx* ctx, Arena& a, const rdx_table& t, int* status, uint32_t* row_bytes,
                          bool in_place) {
  rdx::DevTable d{};
  d.layout = t.layout;
  d.sh_degree = t.sh_degree;
  d.color_dtype = t.color_dtype;
  d.sh_codec = t.sh_codec;
  const uint64_t n = t.count;
  const TableBytes b = table_bytes(t, n);
  *row_bytes = 0;
  if (t.layout == RDX_LAYOUT_RAW) {
    d.centers = stage_column(ctx, a, t.centers, b.centers, 4, status);
    d.log_scales = stage_column(ctx, a, t.log_scales, b.scales, 4, status);
    d.quats = stage_column(ctx, a, t.quats, b.quats, 16, status);
    d.opacities = stage_column(ctx, a, t.opacities, b.opacities, 4, status);
    // colour rows in place where a kernel flavour stages them in whole 16-byte pieces
    d.colors = stage_column(ctx, a, reinterpret_cast<const char*>(t.colors), b.colors, color_vec_bytes(t), status,
                            in_place && rdx::project_host_rows_supported(d), n, row_bytes);
    return d;
  }
  if (t.layout == RDX_LAYOUT_PACKED) {
    d.packed = stage_column(ctx, a, t.packed, b.words, 16, status);
    for (int c = 0; c < 4; c++) d.packed_encoding[c] = t.packed_encoding[c];
  } else {
    d.ext_a = stage_column(ctx, a, t.ext_a, b.words, 16, status);
    d.ext_b = stage_column(ctx, a, t.ext_b, b.words, 16, status);
  }
  if (t.sh_palette) {
    d.sh_palette = stage_column(ctx, a, t.sh_palette, (size_t)t.sh_palette_size * t.sh_stride * 16, 16, status);
    d.sh_label = stage_column(ctx, a, t.sh_label, n * 2, 2, status);
    d.sh_stride = t.sh_stride;
    d.sh_palette_size = t.sh_palette_size;
  } else {
    for (size_t c = 0; c < b.sh_texels; c++) d.ext_sh[c] = stage_column(ctx, a, t.ext_sh[c], b.words, 16, status);
  }
  return d;
}

// Every column of the table is device memory
bool all_device(const rdx_table& t) {
  if (t.layout == RDX_LAYOUT_RAW) {
    for (const void* p : {(const void*)t.centers, (const void*)t.log_scales, (const void*)t.quats,
                          (const void*)t.opacities, t.colors})
      if (!is_device_ptr(p)) return false;
    return true;
  }
  if (t.layout == RDX_LAYOUT_PACKED) {
    if (!is_device_ptr(t.packed)) return false;
  } else if (!is_device_ptr(t.ext_a) || !is_device_ptr(t.ext_b)) {
    return false;
  }
  if (t.sh_palette) return is_device_ptr(t.sh_palette) && is_device_ptr(t.sh_label);
  for (int c = 0; c < sh_texels(t.sh_codec, t.sh_degree); c++)
    if (!is_device_ptr(t.ext_sh[c])) return false;
  return true;
}

rdx::DevParams dev_params(const rdx_params& p) {
  rdx::DevParams d{};
  d.max_std_dev = p.max_std_dev;
  d.min_alpha = p.min_alpha;
  d.blur_amount = p.blur_amount;
  d.pre_blur_amount = p.pre_blur_amount;
  d.clip_xy = p.clip_xy;
  d.min_pixel_radius = p.min_pixel_radius;
  d.max_pixel_radius = p.max_pixel_radius;
  d.min_contribution = p.min_contribution;
  d.focal_distance = p.focal_distance;
  d.aperture_tan = p.aperture_tan;
  d.sort_guard = p.sort_guard;
  d.lod_inflate = p.lod_inflate;
  d.max_sh_degree = p.max_sh_degree;
  return d;
}

// Outputs on the device: the caller's pointers, or staging for host ones
struct OutPlan {
  rdx::ProjOutputs dev{};
  struct Back {
    void* host;
    const void* dev;
    size_t bytes;
  };
  std::vector<Back> back;
};

template <class T>
T* stage_out(rdx_ctx* ctx, Arena& a, T* user, size_t bytes, size_t align, OutPlan& plan, int* status) {
  if (!user) return nullptr;
  if (is_device_ptr(user)) {
    if (!aligned(user, align)) *status = fail(ctx, RDX_ERR_ARG, "a device output is not %zu-byte aligned", align);
    return user;
  }
  T* d = reinterpret_cast<T*>(a.take<char>(bytes));
  if (d) plan.back.push_back({user, d, bytes});
  return d;
}

int copy_back(rdx_ctx* ctx, const OutPlan& plan) {
  for (const auto& b : plan.back) {
    if (b.bytes) RDX_CUDA(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, ctx->stream), "copy of an output");
  }
  return RDX_OK;
}

struct Camera {
  rdx::DevEye eye[2];
  double fh3[2][9];  // from_head 3x3, row-major
};

int check_camera(rdx_ctx* ctx, const rdx_camera* cam) {
  if (!cam) return fail(ctx, RDX_ERR_ARG, "camera is NULL");
  if (cam->eyes < 1 || cam->eyes > 2) return fail(ctx, RDX_ERR_ARG, "SplatCamera: 1 or 2 eyes, not %d", cam->eyes);
  if (!(cam->width > 0) || !(cam->height > 0)) return fail(ctx, RDX_ERR_ARG, "render size %gx%g", cam->width, cam->height);
  return RDX_OK;
}

// SplatCamera.setViews (src/render/splatCamera.ts:119-138) in float64
Camera setup_camera(const rdx_camera& cam) {
  Camera c{};
  double head_world[16];
  mat4_invert(cam.head, head_world);
  for (int v = 0; v < cam.eyes; v++) {
    rdx::DevEye& e = c.eye[v];
    double fh[16];
    // Matrix4.equals: element values (splatCamera.ts:128)
    const bool identity = std::equal(cam.eye[v].view, cam.eye[v].view + 16, cam.head);
    e.identity = identity ? 1 : 0;
    if (identity) {
      memset(fh, 0, sizeof(fh));
      fh[0] = fh[5] = fh[10] = fh[15] = 1.0;
    } else {
      mat4_mul(cam.eye[v].view, head_world, fh);
    }
    for (int r = 0; r < 3; r++) {
      for (int col = 0; col < 4; col++) e.from_head[r * 4 + col] = fh[col * 4 + r];
      for (int col = 0; col < 3; col++) c.fh3[v][r * 3 + col] = fh[col * 4 + r];
    }
    memcpy(e.proj, cam.eye[v].projection, sizeof(e.proj));
    e.focal_d[0] = cam.width * 0.5 * e.proj[0];
    e.focal_d[1] = cam.height * 0.5 * e.proj[5];
    e.proj11 = (float)e.proj[5];
    e.ortho = cam.eye[v].ortho ? 1 : 0;
  }
  return c;
}

// One descriptor: setTransforms (src/render/splatTransform.tsl.ts:78-107) and
// the generator context's view origin (src/gpu/splatGenerator.ts:105-112)
rdx::ProjDesc make_desc(const rdx_camera& cam, const Camera& c, const rdx_object& obj, const rdx::DevTable& table,
                        const rdx_params& params, uint64_t out_offset, uint64_t out_n, int bits, int pass,
                        int cull_keys) {
  rdx::ProjDesc d{};
  d.table = table;
  d.params = dev_params(obj.params ? *obj.params : params);
  double a[16];
  mat4_mul(cam.head, obj.world, a);
  double a3[9];
  bool zero = true;
  for (int r = 0; r < 3; r++) {
    for (int col = 0; col < 4; col++) d.a[r * 4 + col] = a[col * 4 + r];
    for (int col = 0; col < 3; col++) {
      a3[r * 3 + col] = a[col * 4 + r];
      zero = zero && a3[r * 3 + col] == 0.0;
    }
  }
  double inv[16];
  mat4_invert(a, inv);
  d.origin[0] = inv[12];
  d.origin[1] = inv[13];
  d.origin[2] = inv[14];
  d.degenerate = zero ? 1 : 0;
  d.count = obj.count;
  d.out_offset = out_offset;
  d.out_n = out_n;
  for (int v = 0; v < cam.eyes; v++) {
    d.eye[v] = c.eye[v];
    for (int r = 0; r < 3; r++) {
      for (int col = 0; col < 3; col++) {
        double s = c.fh3[v][r * 3 + 0] * a3[0 * 3 + col] + c.fh3[v][r * 3 + 1] * a3[1 * 3 + col] +
                   c.fh3[v][r * 3 + 2] * a3[2 * 3 + col];
        d.eye[v].wd[r * 3 + col] = s;
      }
    }
  }
  d.segment = 0;
  d.width = cam.width;
  d.height = cam.height;
  d.ndc_z_min = cam.ndc_z_min;
  d.eyes = cam.eyes;
  d.sort_bits = bits;
  d.cull_keys = cull_keys;
  d.keys_only = pass == RDX_PASS_KEYS ? 1 : 0;
  return d;
}

// The unit quaternion of a rotation matrix (row-major), by the trace and the
// largest diagonal element (Shoemake's method): the rotation three.js
// Matrix4.decompose gives setTransform (src/render/splatTransform.tsl.ts:64-74)
// and SplatCamera.setViews (src/render/splatCamera.ts:129-131)
void rotation_quat(const double m[9], double q[4]) {
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

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

double det3_cols(const double* c0, const double* c1, const double* c2) {
  return c0[0] * (c1[1] * c2[2] - c1[2] * c2[1]) - c1[0] * (c0[1] * c2[2] - c0[2] * c2[1]) +
         c2[0] * (c0[1] * c1[2] - c0[2] * c1[1]);
}

// Matrix4.decompose's rotation of a column-major 4x4: columns over their
// lengths, the first negated when the determinant is negative
void decompose_rotation(const double m[16], double q[4]) {
  const double* c[3] = {m, m + 4, m + 8};
  double len[3] = {sqrt(dot3(c[0], c[0])), sqrt(dot3(c[1], c[1])), sqrt(dot3(c[2], c[2]))};
  if (det3_cols(c[0], c[1], c[2]) < 0.0) len[0] = -len[0];
  double r[9];
  for (int row = 0; row < 3; row++)
    for (int col = 0; col < 3; col++) r[row * 3 + col] = c[col][row] / len[col];
  rotation_quat(r, q);
}

// isUniformScale (src/render/splatTransform.tsl.ts:46-62): with G = M^T M and
// s2 = trace(G) / 3, every entry of G - s2 I within 1e-6 s2 and det(M) > 0;
// then the rotation and |det(M)|^(1/3) of setTransform (64-74)
bool uniform_transform(const double a[16], double q[4], double* scale) {
  const double* c[3] = {a, a + 4, a + 8};
  const double s2 = (dot3(c[0], c[0]) + dot3(c[1], c[1]) + dot3(c[2], c[2])) / 3.0;
  if (!(s2 > 0)) return false;
  for (int i = 0; i < 3; i++)
    for (int j = i; j < 3; j++)
      if (fabs(dot3(c[i], c[j]) - (i == j ? s2 : 0.0)) > 1e-6 * s2) return false;
  const double det = det3_cols(c[0], c[1], c[2]);
  if (!(det > 0)) return false;
  decompose_rotation(a, q);
  *scale = cbrt(fabs(det));
  return true;
}

// One launch per kind: layout, SH degree and colour type or SH codec (also a tuning key)
int table_kind_of(const rdx_table& t) {
  return t.layout * 100 + t.sh_degree * 10 + (t.layout == RDX_LAYOUT_RAW ? t.color_dtype : t.sh_codec);
}

struct ProjectCall {
  std::vector<rdx::ProjDesc> descs;
  std::vector<int> groups;  // start of each group of one kernel kind in descs (+ end)
  std::vector<uint32_t> group_tiles;
  std::vector<uint64_t> seg_begin, seg_end;  // rows of each view (its sort segment)
  uint64_t n = 0;
};

// One view of a frame: a collection seen by a camera
struct ViewRef {
  const rdx_object* objects;
  int n_objects;
  const rdx_camera* camera;
};

// Descriptors of every (view, object) pair, grouped by kernel kind (one launch
// per kind). View v's rows follow view v-1's; eye e of row r is output
// e * n + r; the keys of view v are sort segment v.
int plan_views(rdx_ctx* ctx, Arena& a, const ViewRef* views, int n_views, const rdx_params* params, int bits, int pass,
               int cull_keys, ProjectCall& call) {
  int status = RDX_OK;
  std::map<const rdx_table*, rdx::DevTable> staged;
  std::map<const rdx_table*, uint32_t> row_bytes;  // of each table's columns read in place
  // rows are read in place only in launches without the sort guard (its kernels stage no rows)
  bool guarded = params->sort_guard > 0.0f;
  for (int v = 0; v < n_views; v++)
    for (int i = 0; i < views[v].n_objects; i++)
      guarded = guarded || (views[v].objects[i].params && views[v].objects[i].params->sort_guard > 0.0f);
  uint64_t n = 0;
  for (int v = 0; v < n_views; v++)
    for (int i = 0; i < views[v].n_objects; i++) n += views[v].objects[i].count;
  call.n = n;
  std::map<int, std::vector<rdx::ProjDesc>> by_kind;
  uint64_t offset = 0;
  for (int v = 0; v < n_views; v++) {
    const ViewRef& vw = views[v];
    const Camera c = setup_camera(*vw.camera);
    call.seg_begin.push_back(offset);
    for (int i = 0; i < vw.n_objects; i++) {
      const rdx_object& o = vw.objects[i];
      const rdx_table& t = *o.table;
      if (!staged.count(o.table)) staged[o.table] = stage_table(ctx, a, t, &status, &row_bytes[o.table], !guarded);
      const int kind = table_kind_of(t);
      if (o.count > 0) {
        rdx::ProjDesc d = make_desc(*vw.camera, c, o, staged[o.table], *params, offset, n, bits, pass, cull_keys);
        d.host_row_bytes = row_bytes[o.table];
        d.segment = v;
        d.object = i;
        by_kind[kind].push_back(d);
      }
      offset += o.count;
    }
    call.seg_end.push_back(offset);
  }
  for (auto& kv : by_kind) {
    call.groups.push_back((int)call.descs.size());
    uint32_t tiles = 0;
    for (auto& d : kv.second) {
      d.first_tile = tiles;
      tiles += (uint32_t)((d.count + rdx::kProjTile - 1) / rdx::kProjTile);
      call.descs.push_back(d);
    }
    call.group_tiles.push_back(tiles);
  }
  call.groups.push_back((int)call.descs.size());
  return status;
}

// Sort tiles of the views' segments (each segment starts a new tile)
uint32_t segment_tiles(const ProjectCall& call, std::vector<uint32_t>* prefix) {
  uint32_t t = 0;
  for (size_t v = 0; v < call.seg_begin.size(); v++) {
    if (prefix) prefix->push_back(t);
    t += tiles_of(call.seg_end[v] - call.seg_begin[v]);
  }
  if (prefix) prefix->push_back(t);
  return t;
}

int check_objects(rdx_ctx* ctx, const rdx_object* objects, int n_objects) {
  if (n_objects < 0 || (n_objects > 0 && !objects)) return fail(ctx, RDX_ERR_ARG, "objects is NULL");
  uint64_t n = 0;
  for (int i = 0; i < n_objects; i++) {
    int s = check_table(ctx, objects[i].table, i);
    if (s != RDX_OK) return s;
    if (objects[i].count > objects[i].table->count)
      return fail(ctx, RDX_ERR_CAPACITY, "object %d draws %llu of its table's %llu splats", i,
                  (unsigned long long)objects[i].count, (unsigned long long)objects[i].table->count);
    n += objects[i].count;
  }
  if (n > rdx::kMaxSegmentKeys) return fail(ctx, RDX_ERR_CAPACITY, "%llu splats (at most %u)", (unsigned long long)n, rdx::kMaxSegmentKeys);
  return RDX_OK;
}

// ---- digit-pass variants (rdx_ctx_set_sort_variant's numbering) and tuning ----

constexpr int kSortVariants = 7;  // 0 onesweep by size, 1-3 cooperative, 4-6 onesweep 4096/2048/1024-key tiles

struct SortPlan {
  int coop = rdx::kCoopNone;
  int pass_items = 0;
};

SortPlan plan_of(int variant) {
  SortPlan p;
  if (variant >= 1 && variant <= 3) p.coop = variant;  // kCoop1024x16, kCoop512x16, kCoop1024x8
  if (variant == 4) p.pass_items = 16;
  if (variant == 5) p.pass_items = 8;
  if (variant == 6) p.pass_items = 4;
  return p;
}

// Whether `variant` can run a sort of `segments` segments of max_tiles
// 4096-key tiles with `lookback_words` lookback words
bool variant_feasible(int variant, int segments, uint32_t max_tiles, int passes, size_t lookback_words) {
  const SortPlan p = plan_of(variant);
  if (p.coop != rdx::kCoopNone) return segments == 1 && rdx::coop_blocks(p.coop) > 0;
  if (p.pass_items) return (size_t)passes * max_tiles * (size_t)(16 / p.pass_items) * rdx::kRadix <= lookback_words;
  return true;
}

// A workload's shape for the tuning cache: sort or frame, key width, one
// segment or many, the key count's power of two and the frame's table kind
uint64_t tune_key(int frame, int bits, int segments, uint64_t n, int table_kind) {
  int log2n = 0;
  while (log2n < 63 && (1ull << log2n) < n) log2n++;
  return ((((uint64_t)frame * 8 + (uint64_t)(bits / 8)) * 2 + (segments > 1 ? 1 : 0)) * 64 + (uint64_t)log2n) * 4096 +
         (uint64_t)(table_kind & 4095);
}

// The digit-pass variant of a sort: the context's forced choice, else a tuned
// one for this shape, else the onesweep passes with tiles by size
int sort_variant(const rdx_ctx* ctx, int segments, uint64_t n, int bits, int frame, int table_kind) {
  if (ctx->sort_variant >= 0) return ctx->sort_variant;
  auto it = ctx->tuned.find(tune_key(frame, bits, segments, n, table_kind));
  if (it != ctx->tuned.end()) return it->second.sort_variant;
  return 0;
}

int project_warps(const rdx_ctx* ctx, int segments, uint64_t n, int bits, int table_kind) {
  auto it = ctx->tuned.find(tune_key(1, bits, segments, n, table_kind));
  return it != ctx->tuned.end() ? it->second.project_warps : 0;
}


// Enqueue one sort (every pass); it takes a fresh lookback epoch on the device
int run_sort(rdx_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
             const SegBufs& sb, int segments, uint32_t max_tiles, int bits, const rdx::SortScratch& sc,
             bool zeroed, uint32_t* visible = nullptr, bool visible_ref = false) {
  const int passes = bits / 8;
  int st = ensure_lookback(ctx, (size_t)passes * lookback_tiles(max_tiles) * rdx::kRadix);
  if (st != RDX_OK) return st;
  rdx::SortCall c{};
  c.keys_in = keys_in;
  c.vals_in = vals_in;
  c.keys_out = keys_out;
  c.vals_out = vals_out;
  c.segs = rdx::SortSegments{sb.begin, sb.end, sb.tiles, segments, max_tiles};
  c.bits = bits;
  c.zeroed = zeroed;
  c.scratch = sc;
  c.lookback = ctx->lookback;
  c.lookback_words = ctx->lookback_words;
  c.epoch = ctx->error_flag + 1;
  c.error_flag = ctx->error_flag;
  c.spin_limit = ctx->spin_limit;
  c.silent_pass = ctx->silent_pass;
  ctx->silent_pass = -1;  // one sort only
  const int variant = sort_variant(ctx, segments, (uint64_t)max_tiles * rdx::kSortTile, bits, 0, 0);
  const SortPlan plan = plan_of(variant);
  c.coop = plan.coop;
  c.pass_items = plan.pass_items;
  c.visible = visible;
  c.visible_ref = visible_ref;
  int launches = 0;
  RDX_CUDA(rdx::sort_segments(c, ctx->stream, &launches), "sort launch");
  ctx->launches += (uint64_t)launches;
  return RDX_OK;
}

bool any_host(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (p && !is_device_ptr(p)) return true;
  return false;
}

}  // namespace

extern "C" {

int rdx_version(void) { return RDX_VERSION; }

void rdx_params_default(rdx_params* p) {
  if (!p) return;
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

int rdx_ctx_create(int device, rdx_ctx** out) {
  if (!out) return RDX_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return RDX_ERR_CUDA;
  }
  rdx_ctx* ctx = new rdx_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->error_flag, 8) != cudaSuccess || cudaMallocHost(&ctx->error_host, 4) != cudaSuccess ||
      cudaMemset(ctx->error_flag, 0, 8) != cudaSuccess || cudaMalloc(&ctx->host_bytes_dev, 8) != cudaSuccess ||
      cudaMemset(ctx->host_bytes_dev, 0, 8) != cudaSuccess || cudaMallocHost(&ctx->ring, kRingBytes) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ring_event, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    rdx_ctx_destroy(ctx);
    return RDX_ERR_CUDA;
  }
  *ctx->error_host = 0;
  ctx->stream = ctx->own_stream;
  *out = ctx;
  return RDX_OK;
}

int rdx_ctx_destroy(rdx_ctx* ctx) {
  if (!ctx) return RDX_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->lookback) cudaFree(ctx->lookback);
  if (ctx->error_flag) cudaFree(ctx->error_flag);
  if (ctx->host_bytes_dev) cudaFree(ctx->host_bytes_dev);
  if (ctx->error_host) cudaFreeHost(ctx->error_host);
  for (auto& p : ctx->pending) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->ring_event) cudaEventDestroy(ctx->ring_event);
  if (ctx->ring) cudaFreeHost(ctx->ring);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return RDX_OK;
}

int rdx_ctx_set_host_reads(rdx_ctx* ctx, int mode) {
  if (!ctx) return RDX_ERR_ARG;
  if (mode != RDX_HOST_COPY && mode != RDX_HOST_IN_PLACE) return fail(ctx, RDX_ERR_ARG, "host reads: mode %d", mode);
  ctx->host_reads = mode;
  return RDX_OK;
}

int rdx_ctx_host_bytes(rdx_ctx* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  unsigned long long rows = 0;
  RDX_CUDA(cudaMemcpyAsync(&rows, ctx->host_bytes_dev, 8, cudaMemcpyDeviceToHost, ctx->stream), "host bytes");
  RDX_CUDA(cudaMemsetAsync(ctx->host_bytes_dev, 0, 8, ctx->stream), "host bytes");
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  *bytes = ctx->host_bytes + (uint64_t)rows;
  ctx->host_bytes = 0;
  return RDX_OK;
}

int rdx_ctx_set_stream(rdx_ctx* ctx, void* stream) {
  if (!ctx) return RDX_ERR_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return RDX_OK;
}

int rdx_ctx_synchronize(rdx_ctx* ctx) {
  if (!ctx) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  return finish(ctx);
}

int rdx_ctx_reserve(rdx_ctx* ctx, uint64_t max_keys) {
  if (!ctx) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  Arena a(nullptr);
  take_sort_scratch(a, 1, 4, max_keys);
  take_segs(a, 1);
  a.take<uint32_t>(max_keys * 3);  // keys / staged buffers of a frame or splat sort
  int st = ensure_arena(ctx, a.used);
  return st != RDX_OK ? st : ensure_lookback(ctx, (size_t)4 * lookback_tiles(tiles_of(max_keys)) * rdx::kRadix);
}

int rdx_ctx_set_wait(rdx_ctx* ctx, uint32_t polls, int silent_pass) {
  if (!ctx) return RDX_ERR_ARG;
  if (silent_pass >= rdx::kMaxPasses) return fail(ctx, RDX_ERR_ARG, "silent_pass %d (at most %d)", silent_pass, rdx::kMaxPasses - 1);
  ctx->spin_limit = polls;
  ctx->silent_pass = silent_pass < 0 ? -1 : silent_pass;
  return RDX_OK;
}

int rdx_ctx_set_sort_variant(rdx_ctx* ctx, int variant) {
  if (!ctx) return RDX_ERR_ARG;
  if (variant < -1 || variant >= kSortVariants) return fail(ctx, RDX_ERR_ARG, "sort variant %d", variant);
  ctx->sort_variant = variant;
  return RDX_OK;
}

int rdx_ctx_set_profiling(rdx_ctx* ctx, int on) {
  if (!ctx) return RDX_ERR_ARG;
  ctx->profiling = on != 0;
  return RDX_OK;
}

int rdx_ctx_phase_times(rdx_ctx* ctx, double* ms, uint64_t* runs) {
  if (!ctx) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  for (const auto& p : ctx->pending) {
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, p.start, p.stop) == cudaSuccess) {
      ctx->phase_ms[p.phase] += t;
      ctx->phase_runs[p.phase] += 1;
    } else {
      cudaGetLastError();
    }
    ctx->event_pool.push_back(p.start);
    ctx->event_pool.push_back(p.stop);
  }
  ctx->pending.clear();
  for (int i = 0; i < RDX_PHASES; i++) {
    if (ms) ms[i] = ctx->phase_ms[i];
    if (runs) runs[i] = ctx->phase_runs[i];
    ctx->phase_ms[i] = 0.0;
    ctx->phase_runs[i] = 0;
  }
  return RDX_OK;
}

int rdx_ctx_launches(rdx_ctx* ctx, uint64_t* launches) {
  if (!ctx || !launches) return RDX_ERR_ARG;
  *launches = ctx->launches;
  return RDX_OK;
}

const char* rdx_last_error(const rdx_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

int rdx_sort_keys_compute(rdx_ctx* ctx, const double* distances, uint64_t n, int bits, uint32_t* keys) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "SortKeys: bits must be 16, 24 or 32 (got %d)", bits);
  if (n == 0) return RDX_OK;
  if (!distances || !keys) return fail(ctx, RDX_ERR_ARG, "distances or keys is NULL");
  cudaSetDevice(ctx->device);
  const bool host_in = !is_device_ptr(distances), host_out = !is_device_ptr(keys);
  auto layout = [&](Arena& a, const double** d, uint32_t** k) {
    *d = host_in ? a.take<double>(n) : distances;
    *k = host_out ? a.take<uint32_t>(n) : keys;
  };
  Arena dry(nullptr);
  const double* d;
  uint32_t* k;
  layout(dry, &d, &k);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a, &d, &k);
  if (host_in) RDX_CUDA(cudaMemcpyAsync((void*)d, distances, n * 8, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  RDX_CUDA(rdx::launch_keys_f64(d, n, bits, k, ctx->stream), "keys launch");
  ctx->launches += 1;
  if (host_out) RDX_CUDA(cudaMemcpyAsync(keys, k, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return host_in || host_out ? finish(ctx) : RDX_OK;
}

int rdx_sort_keys_compute_f32(rdx_ctx* ctx, const float* distances, uint64_t n, int bits, uint32_t* keys) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "SortKeys: bits must be 16, 24 or 32 (got %d)", bits);
  if (n == 0) return RDX_OK;
  if (!distances || !keys) return fail(ctx, RDX_ERR_ARG, "distances or keys is NULL");
  cudaSetDevice(ctx->device);
  const bool host_in = !is_device_ptr(distances), host_out = !is_device_ptr(keys);
  auto layout = [&](Arena& a, const float** d, uint32_t** k) {
    *d = host_in ? a.take<float>(n) : distances;
    *k = host_out ? a.take<uint32_t>(n) : keys;
  };
  Arena dry(nullptr);
  const float* d;
  uint32_t* k;
  layout(dry, &d, &k);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a, &d, &k);
  if (host_in) RDX_CUDA(cudaMemcpyAsync((void*)d, distances, n * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  RDX_CUDA(rdx::launch_keys_f32(d, n, bits, k, ctx->stream), "keys launch");
  ctx->launches += 1;
  if (host_out) RDX_CUDA(cudaMemcpyAsync(keys, k, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return host_in || host_out ? finish(ctx) : RDX_OK;
}

// The single-segment descriptors of a sort of n keys, written on the device
static int single_segment(rdx_ctx* ctx, const SegBufs& sb, uint64_t n) {
  const uint64_t begin[1] = {0}, end[1] = {n};
  const uint32_t tiles[2] = {0, tiles_of(n)};
  int st = upload(ctx, sb.begin, begin, sizeof(begin));
  if (st == RDX_OK) st = upload(ctx, sb.end, end, sizeof(end));
  return st != RDX_OK ? st : upload(ctx, sb.tiles, tiles, sizeof(tiles));
}

int rdx_sort(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits, uint32_t* ordering, uint64_t ordering_len,
             uint32_t* visible) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "SortKeys.sort: bits must be 16, 24 or 32 (got %d)", bits);
  if (ordering_len < count)
    return fail(ctx, RDX_ERR_CAPACITY, "SortKeys.sort: ordering holds %llu of %llu indices",
                (unsigned long long)ordering_len, (unsigned long long)count);
  if (count > rdx::kMaxSegmentKeys)
    return fail(ctx, RDX_ERR_CAPACITY, "SortKeys.sort: %llu keys (at most %u)", (unsigned long long)count, rdx::kMaxSegmentKeys);
  cudaSetDevice(ctx->device);
  if (count == 0) {
    if (visible) {
      if (is_device_ptr(visible)) {
        RDX_CUDA(cudaMemsetAsync(visible, 0, 4, ctx->stream), "visible");
      } else {
        *visible = 0;
      }
    }
    return RDX_OK;
  }
  if (!keys || !ordering) return fail(ctx, RDX_ERR_ARG, "keys or ordering is NULL");
  const bool host_keys = !is_device_ptr(keys), host_order = !is_device_ptr(ordering);
  const bool host_visible = visible && !is_device_ptr(visible);
  const int passes = bits / 8;
  const uint32_t tiles = tiles_of(count);
  const uint32_t* k;
  uint32_t *o, *vis;
  SegBufs sb;
  rdx::SortScratch sc;
  auto layout = [&](Arena& a) {
    k = host_keys ? a.take<uint32_t>(count) : keys;
    o = host_order ? a.take<uint32_t>(count) : ordering;
    vis = a.take<uint32_t>(1);
    sb = take_segs(a, 1);
    sc = take_sort_scratch(a, 1, passes, count);
  };
  Arena dry(nullptr);
  layout(dry);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (host_keys) RDX_CUDA(cudaMemcpyAsync((void*)k, keys, count * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  s = single_segment(ctx, sb, count);
  if (s != RDX_OK) return s;
  {
    Phase sorting(ctx, RDX_PHASE_SORT);
    s = run_sort(ctx, k, nullptr, nullptr, o, sb, 1, tiles, bits, sc, false, visible ? vis : nullptr, true);
    if (s != RDX_OK) return s;
  }
  if (visible) {
    RDX_CUDA(cudaMemcpyAsync(visible, vis, 4, host_visible ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream),
             "visible copy");
  }
  if (host_order) RDX_CUDA(cudaMemcpyAsync(ordering, o, count * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return host_keys || host_order || host_visible ? finish(ctx) : RDX_OK;
}

int rdx_sort_pairs(rdx_ctx* ctx, uint32_t* keys, uint32_t* values, uint64_t count, int bits) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "WgpuRadixSort: bits must be 16, 24 or 32 (got %d)", bits);
  if (count == 0) return RDX_OK;  // WgpuRadixSort.ts:119-121
  if (count > rdx::kMaxSegmentKeys)
    return fail(ctx, RDX_ERR_CAPACITY, "WgpuRadixSort: %llu keys (at most %u)", (unsigned long long)count, rdx::kMaxSegmentKeys);
  if (!keys || !values) return fail(ctx, RDX_ERR_ARG, "keys or values is NULL");
  cudaSetDevice(ctx->device);
  const bool host_k = !is_device_ptr(keys), host_v = !is_device_ptr(values);
  const int passes = bits / 8;
  const uint32_t tiles = tiles_of(count);
  uint32_t *k, *v;
  SegBufs sb;
  rdx::SortScratch sc;
  auto layout = [&](Arena& a) {
    k = host_k ? a.take<uint32_t>(count) : keys;
    v = host_v ? a.take<uint32_t>(count) : values;
    sb = take_segs(a, 1);
    sc = take_sort_scratch(a, 1, passes, count);
  };
  Arena dry(nullptr);
  layout(dry);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (host_k) RDX_CUDA(cudaMemcpyAsync(k, keys, count * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  if (host_v) RDX_CUDA(cudaMemcpyAsync(v, values, count * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  s = single_segment(ctx, sb, count);
  if (s != RDX_OK) return s;
  {
    Phase sorting(ctx, RDX_PHASE_SORT);
    s = run_sort(ctx, k, v, k, v, sb, 1, tiles, bits, sc, false);
    if (s != RDX_OK) return s;
  }
  if (host_k) RDX_CUDA(cudaMemcpyAsync(keys, k, count * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  if (host_v) RDX_CUDA(cudaMemcpyAsync(values, v, count * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return host_k || host_v ? finish(ctx) : RDX_OK;
}

int rdx_sort_pairs_indirect(rdx_ctx* ctx, uint32_t* keys, uint32_t* values, const uint32_t* count_dev, uint64_t capacity,
                            int bits) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "WgpuRadixSort: bits must be 16, 24 or 32 (got %d)", bits);
  if (capacity == 0) return RDX_OK;
  if (capacity > rdx::kMaxSegmentKeys)
    return fail(ctx, RDX_ERR_CAPACITY, "WgpuRadixSort: capacity %llu (at most %u)", (unsigned long long)capacity, rdx::kMaxSegmentKeys);
  cudaSetDevice(ctx->device);
  if (!is_device_ptr(keys) || !is_device_ptr(values) || !is_device_ptr(count_dev))
    return fail(ctx, RDX_ERR_ARG, "WgpuRadixSort.sortIndirect: keys, values and count must be device memory");
  const int passes = bits / 8;
  const uint32_t tiles = tiles_of(capacity);
  SegBufs sb;
  rdx::SortScratch sc;
  auto layout = [&](Arena& a) {
    sb = take_segs(a, 1);
    sc = take_sort_scratch(a, 1, passes, capacity);
  };
  Arena dry(nullptr);
  layout(dry);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  Phase sorting(ctx, RDX_PHASE_SORT);
  RDX_CUDA(rdx::launch_indirect_segments(count_dev, capacity, sb.begin, sb.end, sb.tiles, ctx->stream), "segments");
  ctx->launches += 1;
  return run_sort(ctx, keys, values, keys, values, sb, 1, tiles, bits, sc, false);
}

int rdx_compact(rdx_ctx* ctx, const uint32_t* keys, uint64_t n, uint32_t invalid, uint32_t* keys_out,
                uint32_t* values_out, uint32_t* count_out) {
  if (!ctx) return RDX_ERR_ARG;
  if (n > rdx::kMaxSegmentKeys) return fail(ctx, RDX_ERR_CAPACITY, "WgpuCompact: %llu keys", (unsigned long long)n);
  if ((!keys && n) || !keys_out || !values_out || !count_out) return fail(ctx, RDX_ERR_ARG, "a buffer is NULL");
  cudaSetDevice(ctx->device);
  const bool hk = n && !is_device_ptr(keys), hko = !is_device_ptr(keys_out), hvo = !is_device_ptr(values_out),
             hc = !is_device_ptr(count_out);
  const uint32_t* k;
  uint32_t *ko, *vo, *c, *lb;
  auto layout = [&](Arena& a) {
    k = hk ? a.take<uint32_t>(n) : keys;
    ko = hko ? a.take<uint32_t>(n) : keys_out;
    vo = hvo ? a.take<uint32_t>(n) : values_out;
    c = hc ? a.take<uint32_t>(1) : count_out;
    lb = a.take<uint32_t>(n / 4096 + 2);
  };
  Arena dry(nullptr);
  layout(dry);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (hk) RDX_CUDA(cudaMemcpyAsync((void*)k, keys, n * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  RDX_CUDA(rdx::launch_compact(k, n, invalid, ko, vo, c, lb, ctx->error_flag, ctx->stream), "compact launch");
  ctx->launches += n ? 3 : 0;
  if (hc) RDX_CUDA(cudaMemcpyAsync(count_out, c, 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  // only the first *count_out pairs are meaningful: all n are copied, the rest unspecified
  if (hko) RDX_CUDA(cudaMemcpyAsync(keys_out, ko, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  if (hvo) RDX_CUDA(cudaMemcpyAsync(values_out, vo, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return hk || hko || hvo || hc ? finish(ctx) : RDX_OK;
}

int rdx_splat_sort(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits, uint32_t* values, uint32_t* count_out,
                   uint32_t* draw_args) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "WgpuSplatSorter: bits must be 16, 24 or 32 (got %d)", bits);
  if (count > rdx::kMaxSegmentKeys) return fail(ctx, RDX_ERR_CAPACITY, "WgpuSplatSorter: %llu keys", (unsigned long long)count);
  if ((!keys && count) || !values || !count_out) return fail(ctx, RDX_ERR_ARG, "a buffer is NULL");
  cudaSetDevice(ctx->device);
  const bool hk = count && !is_device_ptr(keys), hv = !is_device_ptr(values), hc = !is_device_ptr(count_out),
             ha = draw_args && !is_device_ptr(draw_args);
  const int passes = bits / 8;
  const uint32_t tiles = tiles_of(count);
  const uint32_t* k;
  uint32_t *v, *c, *args;
  SegBufs sb;
  rdx::SortScratch sc;
  auto layout = [&](Arena& a) {
    k = hk ? a.take<uint32_t>(count) : keys;
    v = hv ? a.take<uint32_t>(count) : values;
    c = hc ? a.take<uint32_t>(1) : count_out;
    args = ha ? a.take<uint32_t>(5) : draw_args;
    sb = take_segs(a, 1);
    sc = take_sort_scratch(a, 1, passes, count);
  };
  Arena dry(nullptr);
  layout(dry);
  int s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (hk) RDX_CUDA(cudaMemcpyAsync((void*)k, keys, count * 4, cudaMemcpyHostToDevice, ctx->stream), "copy in");
  // WgpuSplatSorter.ts:64-71 compacts the invalid keys away, then sorts: here the
  // first pass sends them to the tail, so values[0, count) is the same order
  Phase sorting(ctx, RDX_PHASE_SORT);
  if (count > 0) {
    s = single_segment(ctx, sb, count);
    if (s != RDX_OK) return s;
    s = run_sort(ctx, k, nullptr, nullptr, v, sb, 1, tiles, bits, sc, false, c, false);
    if (s != RDX_OK) return s;
  } else {
    RDX_CUDA(cudaMemsetAsync(c, 0, 4, ctx->stream), "count");
  }
  if (args) {
    RDX_CUDA(rdx::launch_draw_args(c, args, ctx->stream), "draw args");
    ctx->launches += 1;
  }
  sorting.end();
  if (hc) RDX_CUDA(cudaMemcpyAsync(count_out, c, 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  if (ha) RDX_CUDA(cudaMemcpyAsync(draw_args, args, 20, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  if (hv && count) RDX_CUDA(cudaMemcpyAsync(values, v, count * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  return hk || hv || hc || ha ? finish(ctx) : RDX_OK;
}

}  // extern "C"

namespace {

// The device side of a planned frame: every pointer its kernels use
struct FrameDev {
  rdx::ProjDesc* descs = nullptr;
  rdx::ProjOutputs out{};
  SegBufs sb{};
  rdx::SortScratch sc{};
  uint32_t* ord = nullptr;
  uint32_t* vis = nullptr;         // [views]
  uint64_t* lookback = nullptr;
  uint64_t lookback_words = 0;
  uint32_t* error_flag = nullptr;  // word 0: the error flag, word 1: the lookback epoch
  uint32_t spin_limit = 0;         // polls of a bounded wait (0: the default)
  int silent_pass = -1;            // test hook (see rdx_ctx_set_wait)
  int coop = 0;                    // the digit passes' variant (rdx::kCoop*)
  int pass_items = 0;              // onesweep digit-pass tile (keys a thread; 0: by size)
  int proj_warps = 0;              // warps per projection block (0: the default)
};

// Enqueue a planned frame on `stream`: the projection, then the segmented sort
// (its small state zeroed before the projection) and the visible counts. It reads and
// writes no host memory, so the same sequence can be captured in a CUDA graph.
// `timing` (may be null) gets phase timings.
cudaError_t enqueue_frame(rdx_ctx* timing, const ProjectCall& call, const FrameDev& fd, int bits, bool sort,
                          cudaStream_t stream, uint64_t* launches) {
  const int views = (int)call.seg_begin.size();
  const int passes = bits / 8;
  const bool sorting = sort && call.n > 0;
  cudaError_t e;
  {
    Phase projecting(timing, RDX_PHASE_PROJECT);
    for (size_t g = 0; g + 1 < call.groups.size(); g++) {
      const int start = call.groups[g];
      const int count = call.groups[g + 1] - start;
      // the first launch zeroes the sort's small state (hist, counts, counters)
      rdx::ProjOutputs out = fd.out;
      out.zero = sorting && g == 0 ? fd.sc.hist : nullptr;
      out.zero_words = out.zero ? rdx::sort_small_state_words(views, passes, segment_tiles(call, nullptr)) : 0;
      e = rdx::launch_project(fd.descs + start, call.descs.data() + start, count, call.group_tiles[g], out,
                              fd.error_flag, stream, fd.proj_warps);
      if (e != cudaSuccess) return e;
      if (call.group_tiles[g]) *launches += 1;
    }
  }
  if (sorting) {
    Phase sorting_phase(timing, RDX_PHASE_SORT);
    rdx::SortCall c{};
    c.keys_in = fd.out.keys;
    c.vals_out = fd.ord;
    c.segs = rdx::SortSegments{fd.sb.begin, fd.sb.end, fd.sb.tiles, views, segment_tiles(call, nullptr)};
    c.bits = bits;
    c.zeroed = true;  // zeroed before the projection, so the projection and the sort's kernels run back to back
    c.scratch = fd.sc;
    c.lookback = fd.lookback;
    c.lookback_words = fd.lookback_words;
    c.epoch = fd.error_flag + 1;
    c.error_flag = fd.error_flag;
    c.spin_limit = fd.spin_limit;
    c.silent_pass = fd.silent_pass;
    c.coop = fd.coop;
    c.pass_items = fd.pass_items;
    c.visible = fd.vis;
    int n_launch = 0;
    e = rdx::sort_segments(c, stream, &n_launch);
    *launches += (uint64_t)n_launch;
    if (e != cudaSuccess) return e;
  } else if (sort && fd.vis) {
    e = cudaMemsetAsync(fd.vis, 0, (size_t)views * 4, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The table kind of a frame's first object (0: no objects): a tuning key
int first_table_kind(const ViewRef* views, int n_views) {
  for (int v = 0; v < n_views; v++)
    if (views[v].n_objects > 0) return table_kind_of(*views[v].objects[0].table);
  return 0;
}

// Argument checks shared by the frame entry points; *n = rows of all views
int check_views(rdx_ctx* ctx, const ViewRef* views, int n_views, int sort_bits, int pass, uint64_t* n) {
  if (!valid_bits(sort_bits)) return fail(ctx, RDX_ERR_ARG, "sortBits must be 16, 24 or 32 (got %d)", sort_bits);
  if (pass != RDX_PASS_FULL && pass != RDX_PASS_KEYS) return fail(ctx, RDX_ERR_ARG, "pass %d", pass);
  if (n_views < 1 || !views) return fail(ctx, RDX_ERR_ARG, "no views");
  *n = 0;
  for (int v = 0; v < n_views; v++) {
    int s = check_camera(ctx, views[v].camera);
    if (s != RDX_OK) return s;
    if (views[v].camera->eyes != views[0].camera->eyes)
      return fail(ctx, RDX_ERR_ARG, "view %d has %d eyes, view 0 has %d: a batch shares one eye count", v,
                  views[v].camera->eyes, views[0].camera->eyes);
    s = check_objects(ctx, views[v].objects, views[v].n_objects);
    if (s != RDX_OK) return s;
    for (int i = 0; i < views[v].n_objects; i++) *n += views[v].objects[i].count;
  }
  return RDX_OK;
}

// Segment descriptors of the views' keys, uploaded through the ring
int frame_common(rdx_ctx* ctx, const ViewRef* views, int n_views, const rdx_params* params, int sort_bits, int pass,
                 int cull_keys, const rdx_outputs* out, uint32_t* ordering, uint32_t* visible, bool sort) {
  if (!ctx) return RDX_ERR_ARG;
  uint64_t n = 0;
  int s = check_views(ctx, views, n_views, sort_bits, pass, &n);
  if (s != RDX_OK) return s;
  rdx_params defaults;
  rdx_params_default(&defaults);
  const rdx_params* prm = params ? params : &defaults;
  rdx_outputs none{};
  const rdx_outputs* o = out ? out : &none;
  cudaSetDevice(ctx->device);
  const uint64_t E = (uint64_t)views[0].camera->eyes;
  const int passes = sort_bits / 8;
  if (sort && n > 0 && !ordering) return fail(ctx, RDX_ERR_ARG, "ordering is NULL");
  const bool host_order = sort && ordering && !is_device_ptr(ordering);
  const bool host_visible = sort && visible && !is_device_ptr(visible);

  int status = RDX_OK;
  ProjectCall call;
  OutPlan plan;
  FrameDev fd;
  // Descriptors and segment tables share one block, uploaded in one copy:
  // descs | begin [views] | end [views] | tiles [views + 1], each 256-aligned
  const auto align256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t off_begin = 0, off_end = 0, off_tiles = 0, block_bytes = 0;
  char* block = nullptr;
  auto layout = [&](Arena& a) {
    call = ProjectCall();
    plan = OutPlan();
    fd = FrameDev();
    status = plan_views(ctx, a, views, n_views, prm, sort_bits, pass, cull_keys, call);
    off_begin = align256(call.descs.size() * sizeof(rdx::ProjDesc));
    off_end = off_begin + align256((size_t)n_views * 8);
    off_tiles = off_end + align256((size_t)n_views * 8);
    block_bytes = sort ? off_tiles + ((size_t)n_views + 1) * 4 : off_begin;
    block = a.take<char>(block_bytes);
    fd.descs = reinterpret_cast<rdx::ProjDesc*>(block);
    rdx::ProjOutputs& d = plan.dev;
    if (pass == RDX_PASS_FULL) {
      d.mean2d = stage_out(ctx, a, o->mean2d, E * n * 8, 8, plan, &status);
      d.conic = stage_out(ctx, a, o->conic, E * n * 12, 4, plan, &status);
      d.depth = stage_out(ctx, a, o->depth, E * n * 4, 4, plan, &status);
      d.opacity = stage_out(ctx, a, o->opacity, E * n * 4, 4, plan, &status);
      d.rgb = stage_out(ctx, a, o->rgb, E * n * 12, 4, plan, &status);
      d.radii = stage_out(ctx, a, o->radii, E * n * 12, 4, plan, &status);
      d.words = stage_out(ctx, a, o->words, E * n * 16, 16, plan, &status);
    }
    d.keys = stage_out(ctx, a, o->keys, n * 4, 4, plan, &status);
    d.host_bytes = ctx->host_bytes_dev;
    if (sort) {
      if (!d.keys) d.keys = a.take<uint32_t>(n);
      fd.ord = host_order ? a.take<uint32_t>(n) : ordering;
      fd.vis = a.take<uint32_t>((size_t)n_views);
      fd.sb = SegBufs{reinterpret_cast<uint64_t*>(block + off_begin), reinterpret_cast<uint64_t*>(block + off_end),
                      reinterpret_cast<uint32_t*>(block + off_tiles)};
      fd.sc = take_sort_scratch(a, n_views, passes, n);
    }
    fd.out = d;
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  {
    Phase copying(ctx, RDX_PHASE_COPY_IN);  // staging copies of host tables are issued by layout()
    layout(a);
  }
  if (status != RDX_OK) return status;
  if (sort && n > 0) {
    s = ensure_lookback(ctx, (size_t)passes * lookback_tiles(segment_tiles(call, nullptr)) * rdx::kRadix);
    if (s != RDX_OK) return s;
  }
  if (block_bytes && (!call.descs.empty() || (sort && n > 0))) {
    std::vector<char> host(block_bytes, 0);
    memcpy(host.data(), call.descs.data(), call.descs.size() * sizeof(rdx::ProjDesc));
    if (sort) {
      std::vector<uint32_t> tiles;
      segment_tiles(call, &tiles);
      memcpy(host.data() + off_begin, call.seg_begin.data(), (size_t)n_views * 8);
      memcpy(host.data() + off_end, call.seg_end.data(), (size_t)n_views * 8);
      memcpy(host.data() + off_tiles, tiles.data(), ((size_t)n_views + 1) * 4);
    }
    s = upload(ctx, block, host.data(), block_bytes);
    if (s != RDX_OK) return s;
  }
  fd.lookback = ctx->lookback;
  fd.lookback_words = ctx->lookback_words;
  fd.error_flag = ctx->error_flag;
  fd.spin_limit = ctx->spin_limit;
  {
    const int kind = first_table_kind(views, n_views);
    const SortPlan plan = plan_of(sort_variant(ctx, n_views, n, sort_bits, 1, kind));
    fd.coop = plan.coop;
    fd.pass_items = plan.pass_items;
    fd.proj_warps = project_warps(ctx, n_views, n, sort_bits, kind);
  }
  if (sort && n > 0) {
    fd.silent_pass = ctx->silent_pass;
    ctx->silent_pass = -1;  // one sort only
  }
  RDX_CUDA(enqueue_frame(ctx, call, fd, sort_bits, sort, ctx->stream, &ctx->launches), "frame launch");
  if (sort && visible) {
    RDX_CUDA(cudaMemcpyAsync(visible, fd.vis, (size_t)n_views * 4,
                             host_visible ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream),
             "visible copy");
  }
  Phase copying_out(ctx, RDX_PHASE_COPY_OUT);
  s = copy_back(ctx, plan);
  if (s != RDX_OK) return s;
  if (host_order && n) RDX_CUDA(cudaMemcpyAsync(ordering, fd.ord, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy out");
  copying_out.end();
  bool host_in = false;
  for (int v = 0; v < n_views && !host_in; v++) {
    for (int i = 0; i < views[v].n_objects && !host_in; i++) {
      const rdx_table& t = *views[v].objects[i].table;
      host_in = !all_device(t);
    }
  }
  return host_in || !plan.back.empty() || host_order || host_visible ? finish(ctx) : RDX_OK;
}

}  // namespace

// A batched frame captured once in a CUDA graph (device memory only)
struct rdx_batch {
  rdx_ctx* ctx = nullptr;
  int bits = 32;
  int eyes = 1;
  std::vector<int> view_objects;             // objects of each view
  std::vector<const rdx_table*> tables;      // of each (view, object)
  std::vector<uint64_t> counts;
  ProjectCall call;
  FrameDev fd;
  char* arena = nullptr;                     // descriptors, segments, sort scratch, keys
  uint64_t* lookback = nullptr;
  uint32_t* words = nullptr;                 // error flag, lookback epoch
  uint32_t* error_host = nullptr;
  rdx::ProjDesc* staging = nullptr;          // pinned copy of the descriptors for updates
  cudaEvent_t staged = nullptr;              // the last update's copy is done
  bool staged_used = false;
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_launches = 0;               // kernels in the graph
  size_t lookback_words = 0;
  int table_kind = 0;                        // of the first object (the tuning key)
  uint64_t n = 0;                            // rows of all views
};

namespace {

// Capture the batch's frame (its current plan) in a CUDA graph, replacing any earlier one
int capture_batch(rdx_batch* b) {
  rdx_ctx* ctx = b->ctx;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->graph_launches = 0;
  cudaError_t e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamBeginCapture");
  cudaError_t le = enqueue_frame(nullptr, b->call, b->fd, b->bits, true, b->capture, &b->graph_launches);
  e = cudaStreamEndCapture(b->capture, &b->graph);
  if (le != cudaSuccess) return cuda_fail(ctx, le, "batch capture");
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
  return RDX_OK;
}

void free_batch(rdx_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->capture) cudaStreamDestroy(b->capture);
  if (b->staged) cudaEventDestroy(b->staged);
  if (b->staging) cudaFreeHost(b->staging);
  if (b->error_host) cudaFreeHost(b->error_host);
  if (b->words) cudaFree(b->words);
  if (b->lookback) cudaFree(b->lookback);
  if (b->arena) cudaFree(b->arena);
  delete b;
}

}  // namespace

extern "C" {

int rdx_project(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                const rdx_params* params, int sort_bits, int pass, int cull_keys, const rdx_outputs* out) {
  const ViewRef view{objects, n_objects, camera};
  return frame_common(ctx, &view, 1, params, sort_bits, pass, cull_keys, out, nullptr, nullptr, false);
}

int rdx_frame(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera, const rdx_params* params,
              int sort_bits, const rdx_outputs* out, uint32_t* ordering, uint32_t* visible) {
  const ViewRef view{objects, n_objects, camera};
  return frame_common(ctx, &view, 1, params, sort_bits, RDX_PASS_FULL, 1, out, ordering, visible, true);
}

int rdx_project_backward(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                         const rdx_params* params, const rdx_grads_in* upstream, const rdx_table_grads* grads) {
  if (!ctx) return RDX_ERR_ARG;
  if (!upstream || !grads) return fail(ctx, RDX_ERR_ARG, "upstream or grads is NULL");
  if (!upstream->fwd_opacity) return fail(ctx, RDX_ERR_ARG, "the forward's opacity output is required");
  const ViewRef view{objects, n_objects, camera};
  uint64_t n = 0;
  int s = check_views(ctx, &view, 1, 32, RDX_PASS_FULL, &n);
  if (s != RDX_OK) return s;
  for (int i = 0; i < n_objects; i++) {
    if (objects[i].table->layout != RDX_LAYOUT_RAW)
      return fail(ctx, RDX_ERR_UNSUPPORTED, "object %d: only raw tables have a gradient", i);
    if (!all_device(*objects[i].table)) return fail(ctx, RDX_ERR_ARG, "the gradient takes device memory only (object %d's table)", i);
    const rdx_table_grads& g = grads[i];
    for (const void* p : {(const void*)g.centers, (const void*)g.log_scales, (const void*)g.quats,
                          (const void*)g.opacities, (const void*)g.colors})
      if (p && !is_device_ptr(p)) return fail(ctx, RDX_ERR_ARG, "object %d: a gradient buffer is host memory", i);
    if (g.quats && !aligned(g.quats, 16)) return fail(ctx, RDX_ERR_ARG, "object %d: quats gradient not 16-byte aligned", i);
  }
  for (const void* p : {(const void*)upstream->mean2d, (const void*)upstream->conic, (const void*)upstream->depth,
                        (const void*)upstream->opacity, (const void*)upstream->rgb, (const void*)upstream->fwd_opacity})
    if (p && !is_device_ptr(p)) return fail(ctx, RDX_ERR_ARG, "an upstream gradient is host memory");
  if (n == 0) return RDX_OK;
  rdx_params defaults;
  rdx_params_default(&defaults);
  cudaSetDevice(ctx->device);
  ProjectCall call;
  rdx::ProjDesc* descs = nullptr;
  rdx::GradsOut* gdev = nullptr;
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    call = ProjectCall();
    status = plan_views(ctx, a, &view, 1, params ? params : &defaults, 32, RDX_PASS_FULL, 1, call);
    descs = a.take<rdx::ProjDesc>(call.descs.size());
    gdev = a.take<rdx::GradsOut>(call.descs.size());
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (status != RDX_OK) return status;
  std::vector<rdx::GradsOut> gh;
  for (const rdx::ProjDesc& d : call.descs) {
    const rdx_table_grads& g = grads[d.object];
    gh.push_back(rdx::GradsOut{g.centers, g.log_scales, g.quats, g.opacities, g.colors});
  }
  s = upload(ctx, descs, call.descs.data(), call.descs.size() * sizeof(rdx::ProjDesc));
  if (s == RDX_OK) s = upload(ctx, gdev, gh.data(), gh.size() * sizeof(rdx::GradsOut));
  if (s != RDX_OK) return s;
  const rdx::GradsIn in{upstream->mean2d, upstream->conic, upstream->depth, upstream->opacity, upstream->rgb,
                        upstream->fwd_opacity};
  Phase backward(ctx, RDX_PHASE_PROJECT);
  for (size_t g = 0; g + 1 < call.groups.size(); g++) {
    const int start = call.groups[g];
    const int count = call.groups[g + 1] - start;
    RDX_CUDA(rdx::launch_project_backward(descs + start, gdev + start, call.descs.data() + start, count,
                                          call.group_tiles[g], in, ctx->stream),
             "backward launch");
    if (call.group_tiles[g]) ctx->launches += 1;
  }
  return RDX_OK;
}

int rdx_method_words(int method, int eyes) {
  if (eyes < 1 || eyes > 2) return -1;
  switch (method) {
    case RDX_METHOD_EWA: return 4 * eyes;
    case RDX_METHOD_3DGUT:
    case RDX_METHOD_HTGS: return 6 + 2 * eyes;
    case RDX_METHOD_RAYGS: return 4 + 3 * eyes;
    default: return -1;
  }
}

int rdx_project_words(rdx_ctx* ctx, const rdx_object* objects, int n_objects, const rdx_camera* camera,
                      const rdx_params* params, int method, int sort_bits, int cull_keys, uint32_t* words,
                      uint32_t* keys) {
  if (!ctx) return RDX_ERR_ARG;
  if (method == RDX_METHOD_EWA) {
    rdx_outputs out{};
    out.words = words;
    out.keys = keys;
    return rdx_project(ctx, objects, n_objects, camera, params, sort_bits, RDX_PASS_FULL, cull_keys, &out);
  }
  if (method < RDX_METHOD_3DGUT || method > RDX_METHOD_RAYGS)
    return fail(ctx, RDX_ERR_ARG, "projection method %d (ewa 0, 3dgut 1, htgs 2, raygs 3)", method);
  const ViewRef view{objects, n_objects, camera};
  uint64_t n = 0;
  int s = check_views(ctx, &view, 1, sort_bits, RDX_PASS_FULL, &n);
  if (s != RDX_OK) return s;
  std::vector<rdx::RayDesc> per_object((size_t)std::max(n_objects, 1));
  for (int i = 0; i < n_objects; i++) {
    if (!all_device(*objects[i].table))
      return fail(ctx, RDX_ERR_ARG, "the ray methods take device memory only (object %d's table)", i);
    double a[16];
    mat4_mul(camera->head, objects[i].world, a);
    // other transforms, and cov tables, reach the splat form through the covariance (fromCov)
    per_object[i].uniform = uniform_transform(a, per_object[i].tq, &per_object[i].tscale) ? 1 : 0;
  }
  if ((words && !is_device_ptr(words)) || (keys && !is_device_ptr(keys)))
    return fail(ctx, RDX_ERR_ARG, "the ray methods write device memory only");
  if (n == 0) return RDX_OK;
  for (int v = 0; v < camera->eyes; v++) {
    double fh[16];
    if (std::equal(camera->eye[v].view, camera->eye[v].view + 16, camera->head)) {
      memset(fh, 0, sizeof(fh));
      fh[0] = fh[5] = fh[10] = fh[15] = 1.0;
    } else {
      double head_world[16];
      mat4_invert(camera->head, head_world);
      mat4_mul(camera->eye[v].view, head_world, fh);
    }
    double q[4];
    decompose_rotation(fh, q);
    for (int i = 0; i < n_objects; i++) memcpy(per_object[i].eye_q[v], q, sizeof(q));
  }
  rdx_params defaults;
  rdx_params_default(&defaults);
  cudaSetDevice(ctx->device);
  ProjectCall call;
  rdx::ProjDesc* descs = nullptr;
  rdx::RayDesc* rays = nullptr;
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    call = ProjectCall();
    status = plan_views(ctx, a, &view, 1, params ? params : &defaults, sort_bits, RDX_PASS_FULL, cull_keys, call);
    descs = a.take<rdx::ProjDesc>(call.descs.size());
    rays = a.take<rdx::RayDesc>(call.descs.size());
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (status != RDX_OK) return status;
  std::vector<rdx::RayDesc> rh;
  for (const rdx::ProjDesc& d : call.descs) rh.push_back(per_object[d.object]);
  s = upload(ctx, descs, call.descs.data(), call.descs.size() * sizeof(rdx::ProjDesc));
  if (s == RDX_OK) s = upload(ctx, rays, rh.data(), rh.size() * sizeof(rdx::RayDesc));
  if (s != RDX_OK) return s;
  Phase project(ctx, RDX_PHASE_PROJECT);
  for (size_t g = 0; g + 1 < call.groups.size(); g++) {
    const int start = call.groups[g];
    const int count = call.groups[g + 1] - start;
    RDX_CUDA(rdx::launch_project_rays(descs + start, rays + start, call.descs.data() + start, count,
                                      call.group_tiles[g], method, words, keys, ctx->stream),
             "ray projection launch");
    if (call.group_tiles[g]) ctx->launches += 1;
  }
  return RDX_OK;
}

// The header of a PLY file (host or device bytes) into desc
static int read_ply_header(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx::PlyDesc* d) {
  if (!bytes || nbytes == 0) return fail(ctx, RDX_ERR_ARG, "Invalid PLY header");
  size_t head = (size_t)std::min<uint64_t>(nbytes, 64 * 1024);  // HEADER_MAX_BYTES (ply.ts:16)
  std::vector<unsigned char> buf(head);
  if (is_device_ptr(bytes)) {
    // headers are mostly short: the first 4 KB, and the rest of the 64 KB only
    // when those hold no end_header line (the parser reads up to the first one)
    const size_t all = head;
    head = std::min<size_t>(all, 4096);
    RDX_CUDA(cudaMemcpy(buf.data(), bytes, head, cudaMemcpyDeviceToHost), "PLY header copy");
    const std::string first(reinterpret_cast<const char*>(buf.data()), head);
    if (head < all && first.find("end_header\n") == std::string::npos &&
        first.find("end_header\r\n") == std::string::npos) {
      RDX_CUDA(cudaMemcpy(buf.data() + head, static_cast<const char*>(bytes) + head, all - head,
                          cudaMemcpyDeviceToHost),
               "PLY header copy");
      head = all;
    }
  } else {
    memcpy(buf.data(), bytes, head);
  }
  const char* err = rdx::parse_ply_header(buf.data(), head, nbytes, d);
  return err ? fail(ctx, RDX_ERR_ARG, "%s", err) : RDX_OK;
}

int rdx_ply_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_ply_info* info) {
  if (!ctx || !info) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  rdx::PlyDesc d;
  int s = read_ply_header(ctx, bytes, nbytes, &d);
  if (s != RDX_OK) return s;
  info->count = d.count;
  info->sh_degree = d.sh_degree;
  info->kind = d.kind;
  return RDX_OK;
}

int rdx_decode_ply(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, int sh_degree, float* centers, float* log_scales,
                   float* quats, float* opacities, float* colors) {
  if (!ctx) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  rdx::PlyDesc d;
  int s = read_ply_header(ctx, bytes, nbytes, &d);
  if (s != RDX_OK) return s;
  if (sh_degree < 0) sh_degree = d.sh_degree;
  if (sh_degree > d.sh_degree)
    return fail(ctx, RDX_ERR_ARG, "the file has SH degree %d, not %d", d.sh_degree, sh_degree);
  d.out_degree = sh_degree;
  const uint64_t n = d.count;
  const size_t row = (size_t)(1 + kShCoeffs[sh_degree]) * 3;
  const bool host_in = !is_device_ptr(bytes);
  if (quats && is_device_ptr(quats) && !aligned(quats, 16)) return fail(ctx, RDX_ERR_ARG, "quats is not 16-byte aligned");
  OutPlan plan;
  const unsigned char* dev_bytes = nullptr;
  float *c = nullptr, *l = nullptr, *q = nullptr, *o = nullptr, *col = nullptr;
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    plan = OutPlan();
    dev_bytes = host_in ? a.take<unsigned char>(nbytes) : reinterpret_cast<const unsigned char*>(bytes);
    c = stage_out(ctx, a, centers, n * 12, 4, plan, &status);
    l = stage_out(ctx, a, log_scales, n * 12, 4, plan, &status);
    q = stage_out(ctx, a, quats, n * 16, 16, plan, &status);
    o = stage_out(ctx, a, opacities, n * 4, 4, plan, &status);
    col = stage_out(ctx, a, colors, n * row * 4, 4, plan, &status);
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (status != RDX_OK) return status;
  if (host_in) RDX_CUDA(cudaMemcpyAsync((void*)dev_bytes, bytes, nbytes, cudaMemcpyHostToDevice, ctx->stream), "PLY copy");
  // the header's byte offsets into device addresses
  d.vertex = dev_bytes + (uintptr_t)d.vertex;
  if (d.kind == rdx::kPlyCompressed) {
    d.chunk = dev_bytes + (uintptr_t)d.chunk;
    if (d.sh) d.sh = dev_bytes + (uintptr_t)d.sh;
  }
  {
    Phase decoding(ctx, RDX_PHASE_PROJECT);
    RDX_CUDA(rdx::launch_decode_ply(d, c, l, q, o, col, ctx->stream), "PLY decode launch");
    if (n) ctx->launches += 1;
  }
  s = copy_back(ctx, plan);
  if (s != RDX_OK) return s;
  return host_in || !plan.back.empty() ? finish(ctx) : RDX_OK;
}

static int read_spz_header(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx::SpzDesc* d) {
  if (!bytes || nbytes == 0) return fail(ctx, RDX_ERR_ARG, "Invalid SPZ file");
  if (is_device_ptr(bytes))
    return fail(ctx, RDX_ERR_ARG, "SPZ bytes must be in host memory (the container is unpacked on the host)");
  const char* err = rdx::spz_header(reinterpret_cast<const unsigned char*>(bytes), nbytes, d);
  return err ? fail(ctx, RDX_ERR_ARG, "%s", err) : RDX_OK;
}

int rdx_spz_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_spz_info* info) {
  if (!ctx || !info) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  rdx::SpzDesc d;
  int s = read_spz_header(ctx, bytes, nbytes, &d);
  if (s != RDX_OK) return s;
  info->count = d.count;
  info->version = d.version;
  info->sh_degree = d.sh_degree;
  info->fractional_bits = d.fractional_bits;
  info->flags = d.flags;
  info->container = d.container;
  info->reserved = 0;
  return RDX_OK;
}

int rdx_decode_spz(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, int sh_degree, float* centers, float* log_scales,
                   float* quats, float* opacities, float* colors) {
  if (!ctx) return RDX_ERR_ARG;
  cudaSetDevice(ctx->device);
  rdx::SpzDesc d;
  int s = read_spz_header(ctx, bytes, nbytes, &d);
  if (s != RDX_OK) return s;
  if (sh_degree < 0) sh_degree = d.sh_degree;
  if (sh_degree > d.sh_degree)
    return fail(ctx, RDX_ERR_ARG, "the file has SH degree %d, not %d", d.sh_degree, sh_degree);
  d.out_degree = sh_degree;
  const uint64_t n = d.count;
  const size_t row = (size_t)(1 + kShCoeffs[sh_degree]) * 3;
  if (quats && is_device_ptr(quats) && !aligned(quats, 16)) return fail(ctx, RDX_ERR_ARG, "quats is not 16-byte aligned");
  // The columns unpacked on the host first: a bad stream fails before any device work
  std::unique_ptr<unsigned char[]> payload(new (std::nothrow) unsigned char[d.payload ? d.payload : 1]);
  if (!payload) return fail(ctx, RDX_ERR_NOMEM, "could not allocate %llu bytes for the SPZ columns",
                            (unsigned long long)d.payload);
  const char* err = rdx::spz_unpack(reinterpret_cast<const unsigned char*>(bytes), nbytes, d, payload.get());
  if (err) return fail(ctx, RDX_ERR_ARG, "%s", err);
  OutPlan plan;
  unsigned char* dev_payload = nullptr;
  float *c = nullptr, *l = nullptr, *q = nullptr, *o = nullptr, *col = nullptr;
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    plan = OutPlan();
    dev_payload = a.take<unsigned char>(d.payload);
    c = stage_out(ctx, a, centers, n * 12, 4, plan, &status);
    l = stage_out(ctx, a, log_scales, n * 12, 4, plan, &status);
    q = stage_out(ctx, a, quats, n * 16, 16, plan, &status);
    o = stage_out(ctx, a, opacities, n * 4, 4, plan, &status);
    col = stage_out(ctx, a, colors, n * row * 4, 4, plan, &status);
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (status != RDX_OK) return status;
  // pageable source: the copy has left `payload` when the call returns
  if (d.payload) RDX_CUDA(cudaMemcpyAsync(dev_payload, payload.get(), d.payload, cudaMemcpyHostToDevice, ctx->stream), "SPZ copy");
  d.base = dev_payload;
  {
    Phase decoding(ctx, RDX_PHASE_PROJECT);
    RDX_CUDA(rdx::launch_decode_spz(d, c, l, q, o, col, ctx->stream), "SPZ decode launch");
    if (n) ctx->launches += 1;
  }
  s = copy_back(ctx, plan);
  if (s != RDX_OK) return s;
  return finish(ctx);
}

static int read_rdxfile_header(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx::RdxFile* f) {
  if (!bytes || nbytes == 0) return fail(ctx, RDX_ERR_ARG, "Not an RDX piece of the expected type");
  if (is_device_ptr(bytes))
    return fail(ctx, RDX_ERR_ARG, "RDX bytes must be in host memory (the payloads are inflated on the host)");
  const char* err = rdx::rdxfile_header(reinterpret_cast<const unsigned char*>(bytes), nbytes, f);
  return err ? fail(ctx, RDX_ERR_ARG, "%s", err) : RDX_OK;
}

static int rdxfile_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_rdxfile_info* info,
                             rdx_rdxfile_channel* channels, int capacity, char* header_json, uint64_t json_capacity) {
  cudaSetDevice(ctx->device);
  rdx::RdxFile f;
  int s = read_rdxfile_header(ctx, bytes, nbytes, &f);
  if (s != RDX_OK) return s;
  info->count = f.count;
  info->chunk_size = f.chunk_size;
  info->n_chunks = (int32_t)f.chunk_bytes.size();
  info->n_channels = (int32_t)f.channels.size();
  info->header_json_bytes = f.header_json.size();
  for (int k = 0; channels && k < capacity && k < (int)f.channels.size(); k++) {
    const rdx::RdxChannel& c = f.channels[k];
    if (c.bundle.size() >= sizeof(channels[k].bundle) || c.label.size() >= sizeof(channels[k].label) ||
        c.format.size() >= sizeof(channels[k].format))
      return fail(ctx, RDX_ERR_ARG, "RDX channel name too long: %s.%s", c.bundle.c_str(), c.label.c_str());
    memset(&channels[k], 0, sizeof(channels[k]));
    memcpy(channels[k].bundle, c.bundle.data(), c.bundle.size());
    memcpy(channels[k].label, c.label.data(), c.label.size());
    memcpy(channels[k].format, c.format.data(), c.format.size());
    channels[k].element_bytes = c.element_bytes;
  }
  if (header_json && json_capacity) {
    const size_t nj = std::min<size_t>(f.header_json.size(), json_capacity);
    memcpy(header_json, f.header_json.data(), nj);
  }
  return RDX_OK;
}

// A malformed file may ask for more host memory than there is: no C++
// exception crosses the C ABI, it becomes an error status and text
int rdx_rdxfile_read_info(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, rdx_rdxfile_info* info,
                          rdx_rdxfile_channel* channels, int capacity, char* header_json, uint64_t json_capacity) {
  if (!ctx || !info) return RDX_ERR_ARG;
  try {
    return rdxfile_read_info(ctx, bytes, nbytes, info, channels, capacity, header_json, json_capacity);
  } catch (const std::exception& e) {
    return fail(ctx, RDX_ERR_NOMEM, "RDX header: %s", e.what());
  }
}

static int decode_rdxfile(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, void* const* channels);

int rdx_decode_rdxfile(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, void* const* channels) {
  if (!ctx) return RDX_ERR_ARG;
  try {
    return decode_rdxfile(ctx, bytes, nbytes, channels);
  } catch (const std::exception& e) {
    return fail(ctx, RDX_ERR_NOMEM, "RDX decode: %s", e.what());
  }
}

static int decode_rdxfile(rdx_ctx* ctx, const void* bytes, uint64_t nbytes, void* const* channels) {
  cudaSetDevice(ctx->device);
  rdx::RdxFile f;
  int s = read_rdxfile_header(ctx, bytes, nbytes, &f);
  if (s != RDX_OK) return s;
  const int nc = (int)f.channels.size();
  std::vector<char> wanted(nc > 0 ? nc : 1);
  for (int k = 0; k < nc; k++) wanted[k] = channels && channels[k];
  // Every payload inflated on the host first: a bad chunk fails before any device work
  std::vector<unsigned char> staged;
  std::vector<rdx::RdxSpan> spans;
  static_assert(sizeof(bool) == sizeof(char), "wanted flags");
  const char* err = rdx::rdxfile_unpack(reinterpret_cast<const unsigned char*>(bytes), nbytes, f,
                                        reinterpret_cast<const bool*>(wanted.data()), &staged, &spans);
  if (err) return fail(ctx, RDX_ERR_ARG, "%s", err);
  OutPlan plan;
  std::vector<unsigned char*> outs(nc > 0 ? nc : 1, nullptr);
  unsigned char* dev_staged = nullptr;
  rdx::RdxPiece* dev_pieces = nullptr;
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    plan = OutPlan();
    dev_staged = a.take<unsigned char>(staged.size());
    dev_pieces = a.take<rdx::RdxPiece>(spans.size());
    for (int k = 0; k < nc; k++)
      outs[k] = wanted[k] ? stage_out(ctx, a, reinterpret_cast<unsigned char*>(channels[k]),
                                      f.count * (uint64_t)f.channels[k].element_bytes, 1, plan, &status)
                          : nullptr;
  };
  Arena dry(nullptr);
  layout(dry);
  if (status != RDX_OK) return status;
  s = ensure_arena(ctx, dry.used);
  if (s != RDX_OK) return s;
  Arena a(ctx->arena);
  layout(a);
  if (status != RDX_OK) return status;
  std::vector<rdx::RdxPiece> pieces;
  for (const rdx::RdxSpan& sp : spans)
    pieces.push_back({sp.src, outs[sp.channel] + sp.start * (uint64_t)sp.bytes, sp.count, sp.bytes});
  if (!staged.empty())
    RDX_CUDA(cudaMemcpyAsync(dev_staged, staged.data(), staged.size(), cudaMemcpyHostToDevice, ctx->stream), "RDX copy");
  if (!pieces.empty())
    RDX_CUDA(cudaMemcpyAsync(dev_pieces, pieces.data(), pieces.size() * sizeof(rdx::RdxPiece), cudaMemcpyHostToDevice,
                             ctx->stream),
             "RDX pieces");
  {
    Phase decoding(ctx, RDX_PHASE_PROJECT);
    RDX_CUDA(rdx::launch_untranspose(dev_pieces, pieces.data(), (int)pieces.size(), dev_staged, ctx->stream),
             "RDX transpose launch");
    if (!pieces.empty()) ctx->launches += (uint64_t)((pieces.size() + 65534) / 65535);
  }
  s = copy_back(ctx, plan);
  if (s != RDX_OK) return s;
  return finish(ctx);
}

int rdx_frame_batched(rdx_ctx* ctx, const rdx_view* views, int n_views, const rdx_params* params, int sort_bits,
                      const rdx_outputs* out, uint32_t* ordering, uint32_t* visible) {
  if (!ctx) return RDX_ERR_ARG;
  if (n_views < 1 || !views) return fail(ctx, RDX_ERR_ARG, "no views");
  std::vector<ViewRef> refs;
  for (int v = 0; v < n_views; v++) refs.push_back({views[v].objects, views[v].n_objects, views[v].camera});
  return frame_common(ctx, refs.data(), n_views, params, sort_bits, RDX_PASS_FULL, 1, out, ordering, visible, true);
}

int rdx_batch_create(rdx_ctx* ctx, const rdx_view* views, int n_views, const rdx_params* params, int sort_bits,
                     const rdx_outputs* out, uint32_t* ordering, uint32_t* visible, rdx_batch** batch) {
  if (!ctx || !batch) return RDX_ERR_ARG;
  *batch = nullptr;
  if (n_views < 1 || !views) return fail(ctx, RDX_ERR_ARG, "no views");
  std::vector<ViewRef> refs;
  for (int v = 0; v < n_views; v++) refs.push_back({views[v].objects, views[v].n_objects, views[v].camera});
  uint64_t n = 0;
  int s = check_views(ctx, refs.data(), n_views, sort_bits, RDX_PASS_FULL, &n);
  if (s != RDX_OK) return s;
  if (n == 0) return fail(ctx, RDX_ERR_ARG, "a batch draws no splats");
  cudaSetDevice(ctx->device);
  rdx_outputs none{};
  const rdx_outputs* o = out ? out : &none;
  for (const void* p : {(const void*)o->mean2d, (const void*)o->conic, (const void*)o->depth, (const void*)o->opacity,
                        (const void*)o->rgb, (const void*)o->radii, (const void*)o->words, (const void*)o->keys,
                        (const void*)ordering, (const void*)visible})
    if (p && !is_device_ptr(p)) return fail(ctx, RDX_ERR_ARG, "a batch takes device memory only (an output is host memory)");
  if (!ordering) return fail(ctx, RDX_ERR_ARG, "ordering is NULL");
  for (const ViewRef& r : refs)
    for (int i = 0; i < r.n_objects; i++)
      if (!all_device(*r.objects[i].table)) return fail(ctx, RDX_ERR_ARG, "a batch takes device memory only (a table column is host memory)");
  rdx_params defaults;
  rdx_params_default(&defaults);
  const rdx_params* prm = params ? params : &defaults;
  const uint64_t E = (uint64_t)refs[0].camera->eyes;
  const int passes = sort_bits / 8;

  rdx_batch* b = new rdx_batch();
  b->ctx = ctx;
  b->bits = sort_bits;
  b->eyes = (int)E;
  for (const ViewRef& r : refs) {
    b->view_objects.push_back(r.n_objects);
    for (int i = 0; i < r.n_objects; i++) {
      b->tables.push_back(r.objects[i].table);
      b->counts.push_back(r.objects[i].count);
    }
  }
  int status = RDX_OK;
  auto layout = [&](Arena& a) {
    b->call = ProjectCall();
    b->fd = FrameDev();
    status = plan_views(ctx, a, refs.data(), n_views, prm, sort_bits, RDX_PASS_FULL, 1, b->call);
    FrameDev& fd = b->fd;
    fd.descs = a.take<rdx::ProjDesc>(b->call.descs.size());
    fd.out = rdx::ProjOutputs{o->mean2d, o->conic, o->depth, o->opacity, o->rgb, o->radii, o->words, o->keys};
    if (!fd.out.keys) fd.out.keys = a.take<uint32_t>(n);
    fd.ord = ordering;
    fd.vis = visible ? visible : a.take<uint32_t>((size_t)n_views);
    fd.sb = take_segs(a, n_views);
    fd.sc = take_sort_scratch(a, n_views, passes, n);
  };
  Arena dry(nullptr);
  layout(dry);
  auto bail = [&](int code) {
    free_batch(b);
    return code;
  };
  if (status != RDX_OK) return bail(status);
  const uint32_t max_tiles = segment_tiles(b->call, nullptr);
  const size_t lookback_words = (size_t)passes * lookback_tiles(max_tiles) * rdx::kRadix;
  const size_t ndesc = b->call.descs.size();
  if (cudaMalloc(&b->arena, dry.used + 256) != cudaSuccess || cudaMalloc(&b->lookback, lookback_words * 8) != cudaSuccess ||
      cudaMalloc(&b->words, 8) != cudaSuccess || cudaMallocHost(&b->error_host, 4) != cudaSuccess ||
      cudaMallocHost(&b->staging, ndesc * sizeof(rdx::ProjDesc) + 1) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(ctx, RDX_ERR_NOMEM, "could not allocate a batch's device memory"));
  }
  Arena a(b->arena);
  layout(a);
  if (status != RDX_OK) return bail(status);
  b->fd.lookback = b->lookback;
  b->fd.lookback_words = lookback_words;
  b->fd.error_flag = b->words;
  b->fd.spin_limit = ctx->spin_limit;
  b->table_kind = first_table_kind(refs.data(), n_views);
  b->n = n;
  b->lookback_words = lookback_words;
  {
    const SortPlan plan = plan_of(sort_variant(ctx, n_views, n, sort_bits, 1, b->table_kind));
    b->fd.coop = plan.coop;
    b->fd.pass_items = plan.pass_items;
    b->fd.proj_warps = project_warps(ctx, n_views, n, sort_bits, b->table_kind);
  }
  // descriptors and segments stay in the batch's memory; the graph only reads them
  std::vector<uint32_t> tiles;
  segment_tiles(b->call, &tiles);
  cudaError_t e = cudaMemsetAsync(b->lookback, 0, lookback_words * 8, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->words, 0, 8, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->fd.descs, b->call.descs.data(), ndesc * sizeof(rdx::ProjDesc), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->fd.sb.begin, b->call.seg_begin.data(), (size_t)n_views * 8, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->fd.sb.end, b->call.seg_end.data(), (size_t)n_views * 8, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->fd.sb.tiles, tiles.data(), tiles.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "batch set-up"));
  const int st = capture_batch(b);
  if (st != RDX_OK) return bail(st);
  *batch = b;
  return RDX_OK;
}

int rdx_batch_update(rdx_batch* b, const rdx_view* views, int n_views, const rdx_params* params) {
  if (!b) return RDX_ERR_ARG;
  rdx_ctx* ctx = b->ctx;
  if (!views || n_views != (int)b->view_objects.size())
    return fail(ctx, RDX_ERR_ARG, "a batch update keeps the views (%d, got %d)", (int)b->view_objects.size(), n_views);
  std::vector<ViewRef> refs;
  size_t k = 0;
  for (int v = 0; v < n_views; v++) {
    if (views[v].n_objects != b->view_objects[v]) return fail(ctx, RDX_ERR_ARG, "view %d: the objects changed", v);
    int s = check_camera(ctx, views[v].camera);
    if (s != RDX_OK) return s;
    if (views[v].camera->eyes != b->eyes) return fail(ctx, RDX_ERR_ARG, "view %d: the eye count changed", v);
    for (int i = 0; i < views[v].n_objects; i++, k++) {
      if (views[v].objects[i].table != b->tables[k] || views[v].objects[i].count != b->counts[k])
        return fail(ctx, RDX_ERR_ARG, "view %d object %d: a batch update keeps tables and counts", v, i);
    }
    refs.push_back({views[v].objects, views[v].n_objects, views[v].camera});
  }
  rdx_params defaults;
  rdx_params_default(&defaults);
  ProjectCall call;
  Arena dry(nullptr);
  int s = plan_views(ctx, dry, refs.data(), n_views, params ? params : &defaults, b->bits, RDX_PASS_FULL, 1, call);
  if (s != RDX_OK) return s;
  cudaSetDevice(ctx->device);
  if (b->staged_used) RDX_CUDA(cudaEventSynchronize(b->staged), "batch staging wait");
  const size_t bytes = call.descs.size() * sizeof(rdx::ProjDesc);
  memcpy(b->staging, call.descs.data(), bytes);
  RDX_CUDA(cudaMemcpyAsync(b->fd.descs, b->staging, bytes, cudaMemcpyHostToDevice, ctx->stream), "batch update");
  RDX_CUDA(cudaEventRecord(b->staged, ctx->stream), "batch update event");
  b->staged_used = true;
  b->call.descs = call.descs;
  return RDX_OK;
}

int rdx_batch_launch(rdx_batch* b) {
  if (!b) return RDX_ERR_ARG;
  rdx_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  Phase frame(ctx, RDX_PHASE_BATCH);
  RDX_CUDA(cudaGraphLaunch(b->exec, ctx->stream), "cudaGraphLaunch");
  ctx->launches += b->graph_launches;
  return RDX_OK;
}

int rdx_batch_synchronize(rdx_batch* b) {
  if (!b) return RDX_ERR_ARG;
  rdx_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  RDX_CUDA(cudaMemcpyAsync(b->error_host, b->words, 4, cudaMemcpyDeviceToHost, ctx->stream), "error flag");
  RDX_CUDA(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
  if (*b->error_host) {
    const uint32_t bits = *b->error_host;
    *b->error_host = 0;
    cudaMemsetAsync(b->words, 0, 4, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return device_error(ctx, bits);
  }
  return RDX_OK;
}

int rdx_batch_launches(const rdx_batch* b, uint64_t* launches) {
  if (!b || !launches) return RDX_ERR_ARG;
  *launches = b->graph_launches;
  return RDX_OK;
}

}  // extern "C"

namespace {

// Median milliseconds of `reps` runs of enqueue() on the context's stream
// (one warm-up first), each between its own pair of events
template <class F>
int time_runs(rdx_ctx* ctx, int reps, F&& enqueue, double* ms) {
  std::vector<cudaEvent_t> ev(2 * (size_t)reps + 2, nullptr);
  int st = RDX_OK;
  for (auto& x : ev) {
    if (cudaEventCreate(&x) != cudaSuccess) {
      cudaGetLastError();
      st = fail(ctx, RDX_ERR_CUDA, "tuning events");
      break;
    }
  }
  if (st == RDX_OK) st = enqueue();  // warm-up
  for (int r = 0; r < reps && st == RDX_OK; r++) {
    cudaEventRecord(ev[2 * r], ctx->stream);
    st = enqueue();
    cudaEventRecord(ev[2 * r + 1], ctx->stream);
  }
  std::vector<double> t;
  if (st == RDX_OK && cudaStreamSynchronize(ctx->stream) == cudaSuccess) {
    for (int r = 0; r < reps; r++) {
      float x = 0.0f;
      if (cudaEventElapsedTime(&x, ev[2 * r], ev[2 * r + 1]) == cudaSuccess) t.push_back(x);
    }
  }
  cudaGetLastError();
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  if (st != RDX_OK) return st;
  if (t.empty()) return fail(ctx, RDX_ERR_CUDA, "tuning timings");
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return RDX_OK;
}

void add_candidate(rdx_tune_result* out, int sort_variant, int warps, double ms) {
  if (!out || out->candidates >= RDX_TUNE_MAX) return;
  out->cand_sort[out->candidates] = sort_variant;
  out->cand_warps[out->candidates] = warps;
  out->cand_ms[out->candidates] = ms;
  out->candidates++;
}

}  // namespace

extern "C" {

int rdx_batch_tune(rdx_batch* b, int reps, rdx_tune_result* out) {
  if (!b) return RDX_ERR_ARG;
  rdx_ctx* ctx = b->ctx;
  cudaSetDevice(ctx->device);
  if (reps < 1) reps = 5;
  if (out) memset(out, 0, sizeof(*out));
  const int views = (int)b->view_objects.size();
  const int passes = b->bits / 8;
  const uint32_t max_tiles = segment_tiles(b->call, nullptr);
  FrameDev fd = b->fd;
  auto run = [&]() -> int {
    uint64_t launches = 0;
    cudaError_t e = enqueue_frame(nullptr, b->call, fd, b->bits, true, ctx->stream, &launches);
    return e == cudaSuccess ? RDX_OK : cuda_fail(ctx, e, "tuning frame");
  };
  // The defaults first (onesweep passes with tiles by size, 4-warp projection blocks)
  fd.coop = rdx::kCoopNone;
  fd.pass_items = 0;
  fd.proj_warps = 0;
  double default_ms = 0.0;
  int st = time_runs(ctx, reps, run, &default_ms);
  if (st != RDX_OK) return st;
  add_candidate(out, 0, 4, default_ms);
  // Projection block sizes, with the default sort
  int best_warps = 0;
  double best = default_ms;
  for (int w : {2, 8}) {
    fd.proj_warps = w;
    double ms = 0.0;
    st = time_runs(ctx, reps, run, &ms);
    if (st != RDX_OK) return st;
    add_candidate(out, 0, w, ms);
    if (ms < best) {
      best = ms;
      best_warps = w;
    }
  }
  fd.proj_warps = best_warps;
  // Digit-pass variants, with the chosen projection
  int best_variant = 0;
  for (int v = 1; v < kSortVariants; v++) {
    if (!variant_feasible(v, views, max_tiles, passes, b->lookback_words)) continue;
    const SortPlan p = plan_of(v);
    fd.coop = p.coop;
    fd.pass_items = p.pass_items;
    double ms = 0.0;
    st = time_runs(ctx, reps, run, &ms);
    if (st != RDX_OK) return st;
    add_candidate(out, v, best_warps ? best_warps : 4, ms);
    if (ms < best) {
      best = ms;
      best_variant = v;
    }
  }
  st = rdx_batch_synchronize(b);  // a bounded wait that gave up during tuning
  if (st != RDX_OK) return st;
  const SortPlan p = plan_of(best_variant);
  b->fd.coop = p.coop;
  b->fd.pass_items = p.pass_items;
  b->fd.proj_warps = best_warps;
  ctx->tuned[tune_key(1, b->bits, views, b->n, b->table_kind)] = {best_variant, best_warps};
  st = capture_batch(b);
  if (st != RDX_OK) return st;
  if (out) {
    out->sort_variant = best_variant;
    out->project_warps = best_warps ? best_warps : 4;
    out->default_ms = default_ms;
    out->tuned_ms = best;
  }
  return RDX_OK;
}

int rdx_sort_tune(rdx_ctx* ctx, const uint32_t* keys, uint64_t count, int bits, int reps, rdx_tune_result* out) {
  if (!ctx) return RDX_ERR_ARG;
  if (!valid_bits(bits)) return fail(ctx, RDX_ERR_ARG, "SortKeys.sort: bits must be 16, 24 or 32 (got %d)", bits);
  if (count == 0 || count > rdx::kMaxSegmentKeys) return fail(ctx, RDX_ERR_ARG, "rdx_sort_tune: %llu keys", (unsigned long long)count);
  if (!keys || !is_device_ptr(keys)) return fail(ctx, RDX_ERR_ARG, "rdx_sort_tune takes device keys");
  cudaSetDevice(ctx->device);
  if (reps < 1) reps = 5;
  if (out) memset(out, 0, sizeof(*out));
  const int passes = bits / 8;
  const uint32_t tiles = tiles_of(count);
  uint32_t* o;
  SegBufs sb;
  rdx::SortScratch sc;
  auto layout = [&](Arena& a) {
    o = a.take<uint32_t>(count);
    sb = take_segs(a, 1);
    sc = take_sort_scratch(a, 1, passes, count);
  };
  Arena dry(nullptr);
  layout(dry);
  int st = ensure_arena(ctx, dry.used);
  if (st != RDX_OK) return st;
  st = ensure_lookback(ctx, (size_t)passes * lookback_tiles(tiles) * rdx::kRadix);
  if (st != RDX_OK) return st;
  Arena a(ctx->arena);
  layout(a);
  st = single_segment(ctx, sb, count);
  if (st != RDX_OK) return st;
  const int forced = ctx->sort_variant;
  int best_variant = 0;
  double best = 0.0, default_ms = 0.0;
  for (int v = 0; v < kSortVariants && st == RDX_OK; v++) {
    if (!variant_feasible(v, 1, tiles, passes, ctx->lookback_words)) continue;
    ctx->sort_variant = v;
    double ms = 0.0;
    st = time_runs(ctx, reps, [&]() { return run_sort(ctx, keys, nullptr, nullptr, o, sb, 1, tiles, bits, sc, false); }, &ms);
    if (st != RDX_OK) break;
    add_candidate(out, v, 0, ms);
    if (v == 0) default_ms = ms;
    if (v == 0 || ms < best) {
      best = ms;
      best_variant = v;
    }
  }
  ctx->sort_variant = forced;
  if (st != RDX_OK) return st;
  st = finish(ctx);
  if (st != RDX_OK) return st;
  ctx->tuned[tune_key(0, bits, 1, (uint64_t)tiles * rdx::kSortTile, 0)] = {best_variant, 0};
  if (out) {
    out->sort_variant = best_variant;
    out->default_ms = default_ms;
    out->tuned_ms = best;
  }
  return RDX_OK;
}

int rdx_batch_destroy(rdx_batch* b) {
  if (!b) return RDX_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  free_batch(b);
  return RDX_OK;
}

}  // extern "C"
