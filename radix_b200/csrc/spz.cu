// SPZ files (Niantic's format, as src/core/spz.ts reads it) to raw tables.
// The host unpacks the container: a gzip stream (versions 1 to 4; 4 there is
// version 3's layout) is inflated by zlib up to the end of the SH column,
// SPZ 4's NGSP container has its zstd streams decompressed by libzstd (loaded
// the first time such a file is read), on host threads side by side. The byte
// columns then go to the device, where a warp decodes 32 splats, a lane each
// for the small columns and the whole warp for the colour rows (SpzFile.read,
// src/core/spz.ts:285-348, and decodeSmallestThree, 571-586), into float32
// raw-table columns: float64 arithmetic with every operation explicitly
// rounded, in the order the reference evaluates it, then one rounding to float32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <algorithm>
#include <vector>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr uint32_t kSpzMagic = 0x5053474eu;  // "NGSP" little-endian
// SH coefficient vectors of a degree (SH_VECTORS, spz.ts:54)
__host__ __device__ constexpr int sh_vectors(int degree) {
  return degree <= 0 ? 0 : degree == 1 ? 3 : degree == 2 ? 8 : degree == 3 ? 15 : 24;
}
constexpr int kSpzThreads = 256;
// A warp's staging words: 32 splats' base colour bytes (96) and SH bytes (72 a splat at most)
constexpr uint32_t kSpzColourWords = 32 * 3 / 4;
constexpr uint32_t kSpzStageWords = kSpzColourWords + 32 * 72 / 4;
constexpr int Z_STREAM_END_FINAL = 100;  // the last gzip member ended (not a zlib status)

__host__ __device__ __forceinline__ uint32_t le32(const unsigned char* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }

thread_local char g_error[160];  // the last error text of this thread (each call that fails rewrites it)

const char* error_text(const char* fmt, uint64_t a = 0, uint64_t b = 0) {
  snprintf(g_error, sizeof(g_error), fmt, (unsigned long long)a, (unsigned long long)b);
  return g_error;
}

// Column sizes and offsets of the unpacked payload
void spz_layout(SpzDesc* d) {
  const uint64_t n = d->count;
  const uint64_t sizes[6] = {n * (d->version == 1 ? 6u : 9u), n, n * 3, n * 3, n * (d->version >= 3 ? 4u : 3u),
                             n * (uint64_t)sh_vectors(d->sh_degree) * 3};
  uint64_t at = 0;
  for (int k = 0; k < 6; k++) {
    d->col_off[k] = at;
    d->col_size[k] = sizes[k];
    at += sizes[k];
  }
  d->payload = at;
}

// Inflate a gzip stream (members may be concatenated) into the regions
// out[0] (want[0] bytes), then out[1] (want[1] bytes), stopping when both are
// full: the bytes produced, or a negative value on a bad stream
int64_t gunzip(const unsigned char* in, uint64_t n, unsigned char* const out[2], const uint64_t want[2]) {
  z_stream zs;
  memset(&zs, 0, sizeof(zs));
  if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK) return -1;
  uint64_t in_at = 0, produced = 0;
  int status = Z_OK;
  for (int r = 0; r < 2 && status != Z_STREAM_END_FINAL; r++) {
    uint64_t out_at = 0;
    while (out_at < want[r]) {
      const uint64_t in_chunk = std::min<uint64_t>(n - in_at, 1u << 30);
      const uint64_t out_chunk = std::min<uint64_t>(want[r] - out_at, 1u << 30);
      zs.next_in = const_cast<unsigned char*>(in + in_at);
      zs.avail_in = (uInt)in_chunk;
      zs.next_out = out[r] + out_at;
      zs.avail_out = (uInt)out_chunk;
      status = inflate(&zs, Z_NO_FLUSH);
      in_at += in_chunk - zs.avail_in;
      out_at += out_chunk - zs.avail_out;
      if (status == Z_STREAM_END) {
        // another member follows?
        if (in_at + 2 <= n && in[in_at] == 0x1f && in[in_at + 1] == 0x8b) {
          inflateReset(&zs);
          status = Z_OK;
          continue;
        }
        status = Z_STREAM_END_FINAL;
        break;
      }
      if (status != Z_OK) break;
      if (in_at == n && zs.avail_out != 0) break;  // input exhausted
    }
    produced += out_at;
    if (status != Z_OK && status != Z_STREAM_END_FINAL) break;
  }
  inflateEnd(&zs);
  if (status != Z_OK && status != Z_STREAM_END_FINAL && status != Z_BUF_ERROR) return -2;
  return (int64_t)produced;
}

struct Zstd {
  size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
  unsigned (*is_error)(size_t) = nullptr;
};

const Zstd& zstd() {
  static Zstd z = [] {
    Zstd r;
    void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libzstd.so", RTLD_NOW | RTLD_LOCAL);
    if (h) {
      r.decompress = reinterpret_cast<size_t (*)(void*, size_t, const void*, size_t)>(dlsym(h, "ZSTD_decompress"));
      r.is_error = reinterpret_cast<unsigned (*)(size_t)>(dlsym(h, "ZSTD_isError"));
    }
    return r;
  }();
  return z;
}

// ---- device decode ----

__device__ __forceinline__ double sub(double a, double b) { return __dadd_rn(a, -b); }

__global__ void __launch_bounds__(kSpzThreads) k_decode_spz(SpzDesc d, float* __restrict__ centers,
                                                            float* __restrict__ log_scales, float* __restrict__ quats,
                                                            float* __restrict__ opacities, float* __restrict__ colors) {
  const unsigned char* cen = d.base + d.col_off[0];
  const unsigned char* alp = d.base + d.col_off[1];
  const unsigned char* col = d.base + d.col_off[2];
  const unsigned char* sca = d.base + d.col_off[3];
  const unsigned char* rot = d.base + d.col_off[4];
  const unsigned char* shv = d.base + d.col_off[5];
  // fixed = 1 / (1 << fractionalBits) with a 32-bit shift, as JS evaluates it
  const double fixed = 1.0 / (double)(int32_t)(1u << (d.fractional_bits & 31));
  const double color_scale = 0.28209479177387814 / 0.15;  // SH_C0 / 0.15
  // Every byte-valued column maps one byte (a 9-bit magnitude for version 3
  // rotations) to its value: the block computes each mapping once, with the
  // same rounded operations as for a single splat, and the splats look it up
  __shared__ float s_color[256], s_alpha[256], s_scale[256], s_sh[256];
  __shared__ double s_rot2[256], s_mag[512];
  for (uint32_t b = threadIdx.x; b < 512; b += blockDim.x) {
    if (b < 256) {
      const double x = (double)b;
      s_color[b] = (float)__dadd_rn(__dmul_rn(sub(__ddiv_rn(x, 255.0), 0.5), color_scale), 0.5);
      s_alpha[b] = (float)__ddiv_rn(x, 255.0);
      s_scale[b] = (float)sub(__ddiv_rn(x, 16.0), 10.0);
      s_sh[b] = (float)((x - 128.0) / 128.0);
      s_rot2[b] = sub(__ddiv_rn(x, 127.5), 1.0);
    }
    s_mag[b] = __ddiv_rn((double)b, 511.0);
  }
  __syncthreads();
  __shared__ uint32_t s_stage[kSpzThreads / 32][kSpzStageWords];
  const unsigned char* colour_bytes = reinterpret_cast<const unsigned char*>(s_stage[threadIdx.x >> 5]);
  const unsigned char* sh_bytes = colour_bytes + kSpzColourWords * 4;
  const int file_k = sh_vectors(d.sh_degree), out_k = sh_vectors(d.out_degree);
  const uint32_t row_floats = (uint32_t)(1 + out_k) * 3;
  // row = e / row_floats by a multiply-high (exact for e < 32 rows of at most 75 floats)
  const uint32_t row_magic = (uint32_t)(((1ull << 32) + row_floats - 1) / row_floats);
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  // a warp per 32 splats: a lane per splat for the small columns, the whole
  // warp for the 32 colour rows
  for (uint64_t t = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; t * 32 < d.count; t += warps) {
    const uint64_t i0 = t * 32, i = i0 + lane;
    const uint32_t rows = (uint32_t)min((uint64_t)32, d.count - i0);
    const bool live = i < d.count;
    if (colors) {
      // the warp's colour and SH bytes into shared memory with word loads,
      // then its rows as one span in output order (consecutive lanes write
      // consecutive floats)
      warp_copy_bytes(col + i0 * 3, rows * 3, s_stage[threadIdx.x >> 5], lane);
      warp_copy_bytes(shv + i0 * (uint64_t)file_k * 3, rows * (uint32_t)file_k * 3,
                      s_stage[threadIdx.x >> 5] + kSpzColourWords, lane);
      __syncwarp();
      float* out = colors + i0 * row_floats;
      const uint32_t total = rows * row_floats;
      for (uint32_t e = lane; e < total; e += 32) {
        const uint32_t r = __umulhi(e, row_magic), c = e - r * row_floats;
        out[e] = c < 3 ? s_color[colour_bytes[r * 3 + c]] : s_sh[sh_bytes[r * (uint32_t)file_k * 3 + (c - 3)]];
      }
      __syncwarp();  // before the next tile's bytes replace these
    }
    if (!live) continue;
    // The splat's bytes are all loaded before any of its stores (a float store may
    // alias them as far as the compiler knows, which would order each load
    // after the previous store and so chain their latencies)
    const int cen_bytes = d.version == 1 ? 6 : 9, rot_bytes = d.version >= 3 ? 4 : 3;
    uint32_t cb[9], sb[3], qb[4], ab = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) cb[k] = centers && k < cen_bytes ? cen[i * cen_bytes + k] : 0u;
#pragma unroll
    for (int k = 0; k < 3; k++) sb[k] = log_scales ? sca[i * 3 + k] : 0u;
#pragma unroll
    for (int k = 0; k < 4; k++) qb[k] = quats && k < rot_bytes ? rot[i * rot_bytes + k] : 0u;
    if (opacities) ab = alp[i];
    if (centers) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        double v;
        if (d.version == 1) {
          v = (double)__half2float(__ushort_as_half((unsigned short)(cb[c * 2] | (cb[c * 2 + 1] << 8))));
        } else {
          int32_t code = (int32_t)(cb[c * 3] | (cb[c * 3 + 1] << 8) | (cb[c * 3 + 2] << 16));
          if (code & 0x800000) code -= 0x1000000;
          v = __dmul_rn((double)code, fixed);
        }
        centers[i * 3 + c] = (float)v;
      }
    }
    if (opacities) opacities[i] = s_alpha[ab];
    if (log_scales) {
#pragma unroll
      for (int c = 0; c < 3; c++) log_scales[i * 3 + c] = s_scale[sb[c]];
    }
    if (quats) {
      double q[4];
      if (d.version >= 3) {
        const uint32_t packed = qb[0] | (qb[1] << 8) | (qb[2] << 16) | (qb[3] << 24);
        const int largest = (int)(packed >> 30);
        uint32_t rest = packed;
        double sum = 0.0;
#pragma unroll
        for (int k = 3; k >= 0; k--) {
          if (k == largest) continue;
          const double mag = s_mag[rest & 511u];
          const double v = __dmul_rn(__dmul_rn(0.7071067811865476, mag), (rest >> 9) & 1u ? -1.0 : 1.0);
          rest >>= 10;
          q[k] = v;
          sum = __dadd_rn(sum, __dmul_rn(v, v));
        }
        const double w = __dsqrt_rn(fmax(sub(1.0, sum), 0.0));
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (k == largest) q[k] = w;
      } else {
#pragma unroll
        for (int c = 0; c < 3; c++) q[c] = s_rot2[qb[c]];
        q[3] = __dsqrt_rn(
            fmax(0.0, sub(sub(sub(1.0, __dmul_rn(q[0], q[0])), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]))));
      }
      // normalised, as raw tables hold them
      const double l2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2])),
                                  __dmul_rn(q[3], q[3]));
      float4 out = make_float4(0.f, 0.f, 0.f, 1.f);
      if (l2 > 0.0) {
        const double inv = __ddiv_rn(1.0, __dsqrt_rn(l2));
        out = make_float4((float)__dmul_rn(q[0], inv), (float)__dmul_rn(q[1], inv), (float)__dmul_rn(q[2], inv),
                          (float)__dmul_rn(q[3], inv));
      }
      reinterpret_cast<float4*>(quats)[i] = out;
    }
  }
}

}  // namespace

const char* spz_header(const unsigned char* bytes, uint64_t nbytes, SpzDesc* d) {
  *d = SpzDesc();
  if (!bytes || nbytes < 4) return "Invalid SPZ file";
  if (le32(bytes) == kSpzMagic) {
    // SPZ 4: a plaintext 32-byte header, records, a table of contents, zstd streams
    if (nbytes < 32) return "SPZ file ended unexpectedly";
    d->container = kSpzNgsp;
    d->version = (int)le32(bytes + 4);
    d->count = le32(bytes + 8);
    d->sh_degree = bytes[12];
    d->fractional_bits = bytes[13];
    d->flags = bytes[14];
    d->n_streams = bytes[15];
    d->toc_at = le32(bytes + 16);
    if (d->version != 4) return error_text("Unsupported SPZ version %llu in the NGSP container", (uint64_t)d->version);
    if (d->sh_degree > 4) return error_text("Unsupported SPZ version %llu or SH degree %llu", (uint64_t)d->version, (uint64_t)d->sh_degree);
    if (d->count > 0x7fffffffu) return error_text("Invalid SPZ point count %llu", d->count);
    if (d->toc_at < 32) return "SPZ 4 table of contents inside the header";
    spz_layout(d);
    int present = 0;
    for (int k = 0; k < 6; k++) present += d->col_size[k] > 0;
    if (d->n_streams != present)
      return error_text("SPZ 4 file with %llu streams, %llu expected", (uint64_t)d->n_streams, (uint64_t)present);
    if (d->toc_at + (uint64_t)d->n_streams * 16 > nbytes) return "SPZ file ended unexpectedly";
    uint64_t total = d->toc_at + (uint64_t)d->n_streams * 16;
    int k = 0;
    for (int s = 0; s < d->n_streams; s++) {
      while (d->col_size[k] == 0) k++;
      const unsigned char* e = bytes + d->toc_at + (uint64_t)s * 16;
      const uint32_t low = le32(e), high = le32(e + 4), size_low = le32(e + 8), size_high = le32(e + 12);
      if (high >= (1u << 21) || size_high != 0 || size_low != d->col_size[k])
        return error_text("SPZ 4 stream %llu sizes don't match its header", (uint64_t)s);
      total += ((uint64_t)high << 32) | low;
      k++;
    }
    if (d->count * 9 > total * 1024) return error_text("Invalid SPZ point count %llu for %llu bytes", d->count, total);
    if (total > nbytes) return "SPZ file ended unexpectedly";
    if (total < nbytes) return "SPZ 4 file has bytes after its last stream";
    return nullptr;
  }
  if (bytes[0] != 0x1f || bytes[1] != 0x8b) return "Invalid SPZ file";
  unsigned char head[16];
  unsigned char* const out[2] = {head, nullptr};
  const uint64_t want[2] = {16, 0};
  const int64_t got = gunzip(bytes, nbytes, out, want);
  if (got < 0) return "Invalid SPZ file";
  if (got < 16) return "SPZ file ended unexpectedly";
  if (le32(head) != kSpzMagic) return "Invalid SPZ file";
  d->container = kSpzGzip;
  d->version = (int)le32(head + 4);
  d->count = le32(head + 8);
  d->sh_degree = head[12];
  d->fractional_bits = head[13];
  d->flags = head[14];
  if (d->version < 1 || d->version > 4 || d->sh_degree > 4)
    return error_text("Unsupported SPZ version %llu or SH degree %llu", (uint64_t)d->version, (uint64_t)d->sh_degree);
  spz_layout(d);
  return nullptr;
}

const char* spz_unpack(const unsigned char* bytes, uint64_t nbytes, const SpzDesc& d, unsigned char* payload) {
  if (d.container == kSpzGzip) {
    // the 16-byte header, then the columns straight into payload; what follows
    // the SH (trailers, records) is not read
    unsigned char head[16];
    unsigned char* const out[2] = {head, payload};
    const uint64_t want[2] = {16, d.payload};
    const int64_t got = gunzip(bytes, nbytes, out, want);
    if (got < 0) return "Invalid SPZ file";
    if ((uint64_t)got < 16 + d.payload) return "SPZ file ended unexpectedly";
    return nullptr;
  }
  const Zstd& z = zstd();
  if (!z.decompress || !z.is_error) return "SPZ 4 files need libzstd (libzstd.so.1 was not found)";
  // the streams (one a present column) decompressed side by side on host threads
  struct Stream {
    uint64_t at, comp;
    int column;
  };
  std::vector<Stream> streams;
  uint64_t at = d.toc_at + (uint64_t)d.n_streams * 16, packed = 0;
  int k = 0;
  for (int s = 0; s < d.n_streams; s++) {
    while (d.col_size[k] == 0) k++;
    const unsigned char* e = bytes + d.toc_at + (uint64_t)s * 16;
    const uint64_t comp = ((uint64_t)le32(e + 4) << 32) | le32(e);
    streams.push_back({at, comp, k});
    at += comp;
    packed += comp;
    k++;
  }
  std::vector<char> ok(streams.size(), 0);
  parallel_for(streams.size(), packed, [&](size_t s) {
    const Stream& st = streams[s];
    const size_t out = z.decompress(payload + d.col_off[st.column], d.col_size[st.column], bytes + st.at, st.comp);
    ok[s] = !z.is_error(out) && out == d.col_size[st.column];
  });
  for (size_t s = 0; s < streams.size(); s++)
    if (!ok[s])
      return error_text("SPZ 4 stream %llu does not decompress to its %llu bytes", (uint64_t)s,
                        d.col_size[streams[s].column]);
  return nullptr;
}

cudaError_t launch_decode_spz(const SpzDesc& d, float* centers, float* log_scales, float* quats, float* opacities,
                              float* colors, cudaStream_t stream) {
  if (d.count == 0) return cudaSuccess;
  // one wave of blocks (each builds its lookup tables once), warps looping over tiles of 32 splats
  int device = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_decode_spz, kSpzThreads, 0);
  const uint64_t wave = (uint64_t)std::max(sms, 1) * (uint64_t)std::max(per_sm, 1);
  const uint64_t blocks = std::min<uint64_t>((d.count + kSpzThreads - 1) / kSpzThreads, wave);
  k_decode_spz<<<(unsigned)blocks, kSpzThreads, 0, stream>>>(d, centers, log_scales, quats, opacities, colors);
  return cudaGetLastError();
}

}  // namespace rdx
