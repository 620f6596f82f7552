// rdx_sort_noalloc: SortKeys.sort for callers that may not allocate GPU memory.
//
// Some hosts own all of the device memory and do not let an embedded library
// allocate: an engine that reserves its GPU memory budget up front, or a
// real-time frame loop where a cudaMalloc (which can synchronise the device)
// would stall the frame. This entry point sorts with scratch that lives in a
// file-scope __device__ array of fixed size instead of memory it allocates:
// it calls no cudaMalloc, cudaFree or other allocating routine. The array is
// part of the library's device image, so every GPU that loads the library
// holds it (about 18 MB) until the process exits.
//
// The caller passes the keys and the ordering (and optionally the visible
// count) in device memory. All calls share the one array, which keeps what
// the last call left in it. The histogram, counters and error flag must start
// at zero: each call clears them. The lookback words and their epoch word are
// never cleared: the array is zero when the library loads, and every call
// advances the epoch, so words of earlier calls never match. Two calls that
// overlap on the GPU (different streams, or different host threads) race on
// that array: issue them one after another.
//
// A bounded device wait that gave up is reported only through *visible
// (0xffffffff): with visible == NULL the call has no way to report it.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/radix_b200.h"
#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr uint64_t kNoAllocMaxKeys = 1ull << 20;
constexpr uint32_t kNoAllocMaxTiles = (uint32_t)(kNoAllocMaxKeys / kSortTile);

// Byte offsets inside the array (every region 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kSmallOff = 0;  // hist, valid, ref_hidden, counters, tile counts (zeroed per call)
constexpr size_t kSmallBytes = align256((size_t)(kMaxPasses * kRadix + 2 + kMaxPasses + 1 + kNoAllocMaxTiles) * 4);
constexpr size_t kSegOff = kSmallOff + kSmallBytes;  // begin, end, tiles[2], vbegin, vend, vtiles[2]
constexpr size_t kSegBytes = 256;
constexpr size_t kFlagOff = kSegOff + kSegBytes;  // error flag, visible, lookback epoch
constexpr size_t kFlagBytes = 256;
constexpr size_t kKeysAOff = kFlagOff + kFlagBytes;
constexpr size_t kKeysBytes = align256(kNoAllocMaxKeys * 4);
constexpr size_t kValsAOff = kKeysAOff + kKeysBytes;
constexpr size_t kKeysBOff = kValsAOff + kKeysBytes;
constexpr size_t kValsBOff = kKeysBOff + kKeysBytes;
constexpr size_t kLookbackOff = kValsBOff + kKeysBytes;  // epoch-tagged words: never cleared
constexpr size_t kLookbackBytes = (size_t)kMaxPasses * kNoAllocMaxTiles * kRadix * 8;
constexpr size_t kScratchBytes = kLookbackOff + kLookbackBytes;

// The scratch. In host code `g_noalloc_scratch` only names the symbol; its
// device address comes from cudaGetSymbolAddress with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];


// Segment descriptors of one n-key sort, and the error flag cleared
__global__ void k_noalloc_prepare(uint64_t* begin, uint64_t* end, uint32_t* tiles, uint64_t n, uint32_t* flag) {
  begin[0] = 0;
  end[0] = n;
  tiles[0] = 0;
  tiles[1] = (uint32_t)((n + kSortTile - 1) / kSortTile);
  *flag = 0;
}

// visible (and the caller's copy of it); all ones when a bounded device wait gave up
__global__ void k_noalloc_finish(const uint32_t* valid, const uint32_t* ref_hidden, uint64_t n, const uint32_t* flag,
                                 uint32_t* visible) {
  *visible = *flag ? 0xffffffffu : (uint32_t)n - *ref_hidden;
  (void)valid;
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace rdx

extern "C" int rdx_sort_noalloc(const uint32_t* keys, uint64_t count, int bits, uint32_t* ordering,
                                uint64_t ordering_len, uint32_t* visible, void* stream) {
  using namespace rdx;
  if (bits != 16 && bits != 24 && bits != 32) return RDX_ERR_ARG;
  if (ordering_len < count) return RDX_ERR_CAPACITY;
  if (count > kNoAllocMaxKeys) return RDX_ERR_CAPACITY;  // beyond the fixed scratch
  cudaStream_t s = (cudaStream_t)stream;
  if (count == 0) {
    if (visible) {
      if (!on_device(visible)) return RDX_ERR_ARG;
      if (cudaMemsetAsync(visible, 0, 4, s) != cudaSuccess) return RDX_ERR_CUDA;
    }
    return RDX_OK;
  }
  if (!keys || !ordering || !on_device(keys) || !on_device(ordering) || (visible && !on_device(visible)))
    return RDX_ERR_ARG;
  // The array's address on the current device, looked up on every call: the
  // lookup allocates nothing, and no cached address can outlive its context
  // (after a cudaDeviceReset the array lives at a new address). The first
  // call on a device loads the library's device code there.
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
    cudaGetLastError();
    return RDX_ERR_CUDA;
  }
  unsigned char* b = reinterpret_cast<unsigned char*>(ptr);
  const int passes = bits / 8;
  SortScratch sc{};
  uint32_t* small = reinterpret_cast<uint32_t*>(b + kSmallOff);
  sc.hist = small;
  sc.valid = small + (size_t)passes * kRadix;
  sc.ref_hidden = sc.valid + 1;
  sc.counters = sc.ref_hidden + 1;
  sc.tile_valid = sc.counters + passes + 1;
  uint64_t* seg64 = reinterpret_cast<uint64_t*>(b + kSegOff);
  uint64_t* begin = seg64;
  uint64_t* end = seg64 + 1;
  sc.vbegin = seg64 + 2;
  sc.vend = seg64 + 3;
  uint32_t* tiles = reinterpret_cast<uint32_t*>(seg64 + 4);
  sc.vtiles = tiles + 2;
  uint32_t* flag = reinterpret_cast<uint32_t*>(b + kFlagOff);
  uint32_t* vis_tmp = flag + 1;
  uint32_t* epoch = flag + 2;  // advanced by the sort on the device; never cleared
  sc.keys_a = reinterpret_cast<uint32_t*>(b + kKeysAOff);
  sc.vals_a = reinterpret_cast<uint32_t*>(b + kValsAOff);
  sc.keys_b = reinterpret_cast<uint32_t*>(b + kKeysBOff);
  sc.vals_b = reinterpret_cast<uint32_t*>(b + kValsBOff);

  k_noalloc_prepare<<<1, 1, 0, s>>>(begin, end, tiles, count, flag);
  if (cudaGetLastError() != cudaSuccess) return RDX_ERR_CUDA;
  SortCall c{};
  c.keys_in = keys;
  c.vals_in = nullptr;
  c.keys_out = nullptr;
  c.vals_out = ordering;
  const uint32_t max_tiles = (uint32_t)((count + kSortTile - 1) / kSortTile);
  c.segs = SortSegments{begin, end, tiles, 1, max_tiles};
  c.bits = bits;
  c.zeroed = false;  // the sort zeroes its small state itself
  c.scratch = sc;
  c.lookback = reinterpret_cast<uint64_t*>(b + kLookbackOff);
  c.lookback_words = kLookbackBytes / 8;
  c.epoch = epoch;
  c.error_flag = flag;
  if (sort_segments(c, s, nullptr) != cudaSuccess) return RDX_ERR_CUDA;
  k_noalloc_finish<<<1, 1, 0, s>>>(sc.valid, sc.ref_hidden, count, flag, visible ? visible : vis_tmp);
  if (cudaGetLastError() != cudaSuccess) return RDX_ERR_CUDA;
  return RDX_OK;
}
