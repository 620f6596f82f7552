// PLY files to raw tables on the device: the splat values of PlyFile.read
// (src/core/ply.ts:58-164) for standard 3DGS files and RGB point clouds, and
// of its compressed reader (ply.ts:170-264, SuperSplat / PlayCanvas chunks),
// written as float32 columns (centres, ln scales, normalised quaternions
// x y z w, opacities, base rgb + SH coefficient-major) instead of Radix's
// quantised layouts. The header is read on the host; on the device a lane
// decodes a splat, in float64, and rounds once to float32 (standard files and
// point clouds a warp of 32 records at a time, staged in shared memory).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "rdx_internal.h"

namespace rdx {

namespace {

constexpr double kShC0 = 0.28209479177387814;  // ply.ts:15
constexpr int kTypeBytes[8] = {1, 1, 2, 2, 4, 4, 4, 8};  // host copy (the header's record sizes)

__device__ __forceinline__ int type_bytes(int t) { return t <= 1 ? 1 : (t <= 3 ? 2 : (t <= 6 ? 4 : 8)); }

// TYPES[type].scale of a normalised read (ply.ts:33-42)
__device__ __forceinline__ double type_scale(int t) {
  switch (t) {
    case 0: return 127.0;
    case 1: return 255.0;
    case 2: return 32767.0;
    case 3: return 65535.0;
    case 4: return 2147483647.0;
    case 5: return 4294967295.0;
    default: return 1.0;
  }
}

// One scalar of a record, in the file's byte order (byte loads: records need not be aligned)
__device__ __forceinline__ double read_value(const unsigned char* rec, PlyProp p, bool little, bool normalized) {
  const unsigned char* at = rec + p.offset;
  const int n = type_bytes(p.type);
  uint64_t bits = 0;
  for (int b = 0; b < n; b++) {
    const uint64_t byte = at[b];
    bits |= little ? byte << (8 * b) : byte << (8 * (n - 1 - b));
  }
  double v;
  switch (p.type) {
    case 0: v = (double)(int8_t)(uint8_t)bits; break;
    case 1: v = (double)(uint8_t)bits; break;
    case 2: v = (double)(int16_t)(uint16_t)bits; break;
    case 3: v = (double)(uint16_t)bits; break;
    case 4: v = (double)(int32_t)(uint32_t)bits; break;
    case 5: v = (double)(uint32_t)bits; break;
    case 6: v = (double)__uint_as_float((uint32_t)bits); break;
    default: v = __longlong_as_double((long long)bits); break;
  }
  return normalized ? v / type_scale(p.type) : v;
}

__device__ __forceinline__ uint32_t read_word(const unsigned char* rec, PlyProp p, bool little) {
  const unsigned char* at = rec + p.offset;
  return little ? (uint32_t)at[0] | ((uint32_t)at[1] << 8) | ((uint32_t)at[2] << 16) | ((uint32_t)at[3] << 24)
                : (uint32_t)at[3] | ((uint32_t)at[2] << 8) | ((uint32_t)at[1] << 16) | ((uint32_t)at[0] << 24);
}

// splat-transform's SH byte over [-4, 4] (ply.ts:267-270)
__device__ __forceinline__ double compressed_sh(uint32_t byte) {
  return ((byte == 0u ? 0.0 : (byte == 255u ? 1.0 : ((double)byte + 0.5) / 256.0)) - 0.5) * 8.0;
}

// SplatMath.normalizeQuat (math.ts:12-27)
__device__ __forceinline__ void normalize_quat(double q[4]) {
  const double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (len > 0.0) {
    for (int k = 0; k < 4; k++) q[k] /= len;
  } else {
    q[0] = q[1] = q[2] = 0.0;
    q[3] = 1.0;
  }
}

// A standard file's or point cloud's splat (ply.ts:58-164) from its record:
// value(p, normalized) reads property p as a double, rest(p) an SH value as
// float32, and put(x, v) takes SH value x (coefficient-major) of the kvals kept
template <class Value, class Rest, class Put>
__device__ __forceinline__ void decode_plain(const PlyDesc& d, int kvals, Value value, Rest rest, Put put, double c[3],
                                             double ls[3], double q[4], double& op, double rgb[3]) {
  for (int k = 0; k < 3; k++) c[k] = value(d.xyz[k], false);
  if (d.kind == kPlyStandard) {
    for (int k = 0; k < 3; k++) ls[k] = value(d.scale[k], false);
    // (rot_1, rot_2, rot_3, rot_0) = (x, y, z, w)
    q[0] = value(d.rot[1], false);
    q[1] = value(d.rot[2], false);
    q[2] = value(d.rot[3], false);
    q[3] = value(d.rot[0], false);
    op = 1.0 / (1.0 + exp(-value(d.opacity, false)));
    for (int k = 0; k < 3; k++) rgb[k] = 0.5 + kShC0 * value(d.color[k], false);
#pragma unroll
    for (int x = 0; x < kvals; x++) put(x, rest(d.rest[x]));
  } else {
    const double point = log(0.001);  // POINT_SCALE (ply.ts:18)
    ls[0] = ls[1] = ls[2] = point;
    q[0] = q[1] = q[2] = 0.0;
    q[3] = 1.0;
    op = d.alpha.offset >= 0 ? value(d.alpha, true) : 1.0;
    for (int k = 0; k < 3; k++) rgb[k] = value(d.color[k], true);
#pragma unroll
    for (int x = 0; x < kvals; x++) put(x, 0.0f);
  }
}

// Any file, one thread per splat reading its record in place (compressed
// files, and records too long to stage)
__global__ void k_decode_ply(const PlyDesc d, float* __restrict__ centers, float* __restrict__ log_scales,
                             float* __restrict__ quats, float* __restrict__ opacities, float* __restrict__ colors) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.count) return;
  const bool little = d.little != 0;
  const int kvals = (d.out_degree == 0 ? 0 : (d.out_degree == 1 ? 3 : (d.out_degree == 2 ? 8 : (d.out_degree == 3 ? 15 : 24)))) * 3;
  const int row = 3 + kvals;
  double c[3], ls[3], q[4], op, rgb[3];
  float* col = colors ? colors + i * (uint64_t)row : nullptr;
  if (d.kind == kPlyCompressed) {
    const unsigned char* v = d.vertex + i * d.record;
    const unsigned char* ch = d.chunk + (i / 256) * d.chunk_record;
    double r[18];
    const double defaults[6] = {0.0, 0.0, 0.0, 1.0, 1.0, 1.0};
    for (int k = 0; k < 18; k++)
      r[k] = d.chunk_prop[k].offset >= 0 ? read_value(ch, d.chunk_prop[k], little, false) : defaults[k >= 12 ? k - 12 : 0];
    const uint32_t p = read_word(v, d.packed[0], little);
    c[0] = r[0] + (r[3] - r[0]) * ((double)((p >> 21) & 2047u) / 2047.0);
    c[1] = r[1] + (r[4] - r[1]) * ((double)((p >> 11) & 1023u) / 1023.0);
    c[2] = r[2] + (r[5] - r[2]) * ((double)(p & 2047u) / 2047.0);
    const uint32_t l = read_word(v, d.packed[2], little);
    ls[0] = r[6] + (r[9] - r[6]) * ((double)((l >> 21) & 2047u) / 2047.0);
    ls[1] = r[7] + (r[10] - r[7]) * ((double)((l >> 11) & 1023u) / 1023.0);
    ls[2] = r[8] + (r[11] - r[8]) * ((double)(l & 2047u) / 2047.0);
    const uint32_t w = read_word(v, d.packed[1], little);
    const double sq = 1.4142135623730951;
    const double a = ((double)((w >> 20) & 1023u) / 1023.0 - 0.5) * sq;
    const double b = ((double)((w >> 10) & 1023u) / 1023.0 - 0.5) * sq;
    const double cc = ((double)(w & 1023u) / 1023.0 - 0.5) * sq;
    const double m = sqrt(fmax(0.0, 1.0 - a * a - b * b - cc * cc));
    const uint32_t largest = w >> 30;
    q[3] = largest == 0u ? m : a;
    q[0] = largest == 0u ? a : (largest == 1u ? m : b);
    q[1] = largest <= 1u ? b : (largest == 2u ? m : cc);
    q[2] = largest <= 2u ? cc : m;
    const uint32_t k = read_word(v, d.packed[3], little);
    rgb[0] = r[12] + (r[15] - r[12]) * ((double)((k >> 24) & 255u) / 255.0);
    rgb[1] = r[13] + (r[16] - r[13]) * ((double)((k >> 16) & 255u) / 255.0);
    rgb[2] = r[14] + (r[17] - r[14]) * ((double)((k >> 8) & 255u) / 255.0);
    op = (double)(k & 255u) / 255.0;
    if (col) {
      const unsigned char* s = d.sh ? d.sh + i * d.sh_record : nullptr;
      for (int x = 0; x < kvals; x++) col[3 + x] = s ? (float)compressed_sh(s[d.sh_byte[x]]) : 0.0f;
    }
  } else {
    const unsigned char* v = d.vertex + i * d.record;
    decode_plain(
        d, kvals, [&](PlyProp p, bool normalized) { return read_value(v, p, little, normalized); },
        [&](PlyProp p) { return (float)read_value(v, p, little, false); },
        [&](int x, float f) {
          if (col) col[3 + x] = f;
        },
        c, ls, q, op, rgb);
  }
  normalize_quat(q);
  if (centers)
    for (int k = 0; k < 3; k++) centers[i * 3 + k] = (float)c[k];
  if (log_scales)
    for (int k = 0; k < 3; k++) log_scales[i * 3 + k] = (float)ls[k];
  if (quats) reinterpret_cast<float4*>(quats)[i] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
  if (opacities) opacities[i] = (float)op;
  if (col)
    for (int k = 0; k < 3; k++) col[k] = (float)rgb[k];
}

constexpr int kRowsThreads = 128;  // 4 warps, each staging 32 records
constexpr uint32_t kRowsMaxRecord = 1024;  // 32 KB of shared memory a warp at most

// One value of a staged record: a float32 word when every property the
// decode reads is an aligned little-endian float32 (WORDS), else bytes
__device__ __forceinline__ double staged_value(const uint32_t* sw, uint32_t base, PlyProp p, bool words, bool little,
                                               bool normalized) {
  if (words) return (double)__uint_as_float(sw[(base + (uint32_t)p.offset) >> 2]);
  return read_value(reinterpret_cast<const unsigned char*>(sw) + base, p, little, normalized);
}

// An SH value as written: the float32 word itself, or the float32 of any other type
__device__ __forceinline__ float staged_float(const uint32_t* sw, uint32_t base, PlyProp p, bool words, bool little) {
  if (words) return __uint_as_float(sw[(base + (uint32_t)p.offset) >> 2]);
  return (float)read_value(reinterpret_cast<const unsigned char*>(sw) + base, p, little, false);
}

// Shared-memory row pitch (floats) of the colour rows: rows of a multiple of 4
// floats are written as 16-byte vectors, an odd number of vectors apart (the 8
// lanes of each store phase then fill distinct banks); other rows an odd
// number of floats apart
template <int ROW>
__host__ __device__ constexpr int row_pitch() {
  return ROW % 4 == 0 ? ((ROW / 4) % 2 == 1 ? ROW : ROW + 4) : (ROW | 1);
}

// Standard files and RGB point clouds, one warp per 32 records: the warp
// copies its records into shared memory with coalesced aligned word loads
// (funnel-shifted when the records start off a word boundary), each lane
// decodes one splat from there, and the colour rows (ROW floats a splat) go
// back through the same shared memory so that the warp writes its 32 rows as
// one contiguous span (16-byte stores when VEC: rows of a multiple of 4
// floats and 16-byte aligned colours). `region` is the words of shared memory
// each warp owns, a multiple of 4: at least 32 records and 32 rows of
// row_pitch<ROW>() words.
template <int ROW>
__global__ void __launch_bounds__(kRowsThreads) k_decode_ply_rows(const PlyDesc d, uint32_t region, bool words,
                                                                  bool vec, float* __restrict__ centers,
                                                                  float* __restrict__ log_scales,
                                                                  float* __restrict__ quats,
                                                                  float* __restrict__ opacities,
                                                                  float* __restrict__ colors) {
  extern __shared__ __align__(16) uint32_t s_words[];
  constexpr int kPitch = row_pitch<ROW>();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t r0 = ((uint64_t)blockIdx.x * (kRowsThreads / 32) + (uint64_t)warp) * 32;
  if (r0 >= d.count) return;  // the whole warp
  const uint32_t rows = (uint32_t)min((uint64_t)32, d.count - r0);
  uint32_t* sw = s_words + (size_t)warp * region;

  // the records' bytes [0, len) into sw
  warp_copy_bytes(d.vertex + r0 * d.record, rows * d.record, sw, (uint32_t)lane);
  __syncwarp();

  const bool live = (uint32_t)lane < rows;
  const uint64_t i = r0 + (uint64_t)lane;
  const bool little = d.little != 0;
  const uint32_t base = (uint32_t)lane * d.record;
  constexpr int kVals = ROW - 3;
  double c[3], ls[3], q[4], op, rgb[3];
  float cv[ROW];
  if (live) {
    decode_plain(
        d, kVals, [&](PlyProp p, bool normalized) { return staged_value(sw, base, p, words, little, normalized); },
        [&](PlyProp p) { return staged_float(sw, base, p, words, little); }, [&](int x, float f) { cv[3 + x] = f; }, c,
        ls, q, op, rgb);
    normalize_quat(q);
    for (int k = 0; k < 3; k++) cv[k] = (float)rgb[k];
    if (centers)
      for (int k = 0; k < 3; k++) centers[i * 3 + k] = (float)c[k];
    if (log_scales)
      for (int k = 0; k < 3; k++) log_scales[i * 3 + k] = (float)ls[k];
    if (quats) reinterpret_cast<float4*>(quats)[i] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    if (opacities) opacities[i] = (float)op;
  }
  if (!colors) return;  // uniform
  __syncwarp();  // every lane has read its record: the rows may overwrite them
  float* srow = reinterpret_cast<float*>(sw);
  if constexpr (ROW % 4 == 0) {
    if (vec) {
      constexpr int kQuads = ROW / 4;
      if (live) {
        float4* r4 = reinterpret_cast<float4*>(srow + lane * kPitch);
#pragma unroll
        for (int k = 0; k < kQuads; k++) r4[k] = make_float4(cv[4 * k], cv[4 * k + 1], cv[4 * k + 2], cv[4 * k + 3]);
      }
      __syncwarp();
      const float4* s4 = reinterpret_cast<const float4*>(srow);
      float4* d4 = reinterpret_cast<float4*>(colors + r0 * ROW);
      const uint32_t total4 = rows * kQuads;
      for (uint32_t j = lane; j < total4; j += 32) {
        const uint32_t r = j / kQuads;
        d4[j] = s4[r * (kPitch / 4) + (j - r * kQuads)];
      }
      return;
    }
  }
  if (live) {
#pragma unroll
    for (int k = 0; k < ROW; k++) srow[lane * kPitch + k] = cv[k];
  }
  __syncwarp();
  float* dst = colors + r0 * ROW;
  const uint32_t total = rows * ROW;
  for (uint32_t j = lane; j < total; j += 32) {
    const uint32_t r = j / ROW;
    dst[j] = srow[r * kPitch + (j - r * ROW)];
  }
}

// Every value the staged decode reads is an aligned little-endian float32
bool all_float_words(const PlyDesc& d) {
  if (!d.little || d.record % 4) return false;
  auto word = [](PlyProp p) { return p.offset < 0 || (p.type == 6 && p.offset % 4 == 0); };
  bool ok = word(d.xyz[0]) && word(d.xyz[1]) && word(d.xyz[2]);
  for (int k = 0; k < 3; k++) ok = ok && word(d.color[k]);
  if (d.kind == kPlyStandard) {
    for (int k = 0; k < 3; k++) ok = ok && word(d.scale[k]);
    for (int k = 0; k < 4; k++) ok = ok && word(d.rot[k]);
    ok = ok && word(d.opacity);
    const int vals = (d.out_degree == 0 ? 0 : (d.out_degree == 1 ? 3 : (d.out_degree == 2 ? 8 : (d.out_degree == 3 ? 15 : 24)))) * 3;
    for (int x = 0; x < vals; x++) ok = ok && word(d.rest[x]);
  } else {
    ok = ok && word(d.alpha);
  }
  return ok;
}

template <int ROW>
cudaError_t launch_rows(const PlyDesc& d, float* centers, float* log_scales, float* quats, float* opacities,
                        float* colors, cudaStream_t stream) {
  const uint32_t record_words = (d.record + 3) / 4;
  const uint32_t region = (std::max<uint32_t>(32 * record_words, 32 * row_pitch<ROW>()) + 3) & ~3u;
  const size_t smem = (size_t)region * 4 * (kRowsThreads / 32);
  cudaError_t e = cudaFuncSetAttribute(k_decode_ply_rows<ROW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint64_t warps = (d.count + 31) / 32;
  const uint64_t blocks = (warps + kRowsThreads / 32 - 1) / (kRowsThreads / 32);
  const bool vec = ROW % 4 == 0 && ((uintptr_t)colors & 15u) == 0;
  k_decode_ply_rows<ROW><<<(unsigned)blocks, kRowsThreads, smem, stream>>>(d, region, all_float_words(d), vec,
                                                                           centers, log_scales, quats, opacities,
                                                                           colors);
  return cudaGetLastError();
}

// ---- the header (ply.ts:362-444) ----

struct Prop {
  std::string name;
  int type;
  bool list;
  int offset;
};

struct Element {
  std::string name;
  uint64_t count;
  std::vector<Prop> props;
  uint32_t record;
};

int ply_type(const std::string& name) {
  static const char* names[8] = {"char", "uchar", "short", "ushort", "int", "uint", "float", "double"};
  static const char* aliases[8] = {"int8", "uint8", "int16", "uint16", "int32", "uint32", "float32", "float64"};
  for (int t = 0; t < 8; t++)
    if (name == names[t] || name == aliases[t]) return t;
  return -1;
}

int shdeg(int rest) { return rest >= 72 ? 4 : rest >= 45 ? 3 : rest >= 24 ? 2 : rest > 0 ? 1 : 0; }

const Prop* find(const Element& e, const std::string& name) {
  for (const Prop& p : e.props)
    if (p.name == name && !p.list) return &p;
  return nullptr;
}

PlyProp pp(const Prop* p) { return p ? PlyProp{p->offset, p->type} : PlyProp{-1, 6}; }

thread_local std::string g_error;

}  // namespace

const char* parse_ply_header(const unsigned char* head, uint64_t head_bytes, uint64_t nbytes, PlyDesc* d) {
  memset(d, 0, sizeof(*d));
  std::string text((const char*)head, (size_t)head_bytes);
  size_t end = text.find("end_header\n");
  size_t end_r = text.find("end_header\r\n");
  if (text.compare(0, 3, "ply") != 0 || (end == std::string::npos && end_r == std::string::npos))
    return "Invalid PLY header";
  uint64_t header_len;
  if (end != std::string::npos && (end_r == std::string::npos || end < end_r)) {
    header_len = end + strlen("end_header\n");
  } else {
    end = end_r;
    header_len = end_r + strlen("end_header\r\n");
  }
  int little = -1;
  std::vector<Element> elements;
  size_t pos = text.find('\n') + 1;
  while (pos < end) {
    size_t nl = text.find('\n', pos);
    std::string line = text.substr(pos, nl - pos);
    pos = nl + 1;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::vector<std::string> f;
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) i++;
      size_t j = i;
      while (j < line.size() && line[j] != ' ' && line[j] != '\t') j++;
      if (j > i) f.push_back(line.substr(i, j - i));
      i = j;
    }
    if (f.empty()) continue;
    if (f[0] == "format") {
      if (f.size() < 2 || (f[1] != "binary_little_endian" && f[1] != "binary_big_endian")) {
        g_error = "Unsupported PLY format " + (f.size() > 1 ? f[1] : std::string());
        return g_error.c_str();
      }
      little = f[1] == "binary_little_endian" ? 1 : 0;
    } else if (f[0] == "element" && f.size() >= 3) {
      elements.push_back(Element{f[1], (uint64_t)strtoull(f[2].c_str(), nullptr, 10), {}, 0});
    } else if (f[0] == "property") {
      if (elements.empty()) return "PLY property outside an element";
      Element& e = elements.back();
      if (f.size() >= 5 && f[1] == "list") {
        e.props.push_back(Prop{f[4], ply_type(f[3]), true, -1});
      } else if (f.size() >= 3) {
        const int t = ply_type(f[1]);
        if (t < 0) {
          g_error = "Unsupported PLY property type " + f[1];
          return g_error.c_str();
        }
        e.props.push_back(Prop{f[2], t, false, (int)e.record});
        e.record += (uint32_t)kTypeBytes[t];
      }
    }
  }
  if (little < 0) return "PLY header has no format line";
  d->little = little;
  auto offset_of = [&](const Element* el, uint64_t* out) -> const char* {
    uint64_t off = header_len;
    for (const Element& b : elements) {
      if (&b == el) break;
      for (const Prop& p : b.props)
        if (p.list) {
          g_error = "PLY element " + b.name + " before " + el->name + " has list properties";
          return g_error.c_str();
        }
      // each product checked by a division first, so no count wraps past the file's end
      if (off > nbytes || (b.record && b.count > (nbytes - off) / b.record)) return "PLY file ended unexpectedly";
      off += b.count * b.record;
    }
    if (off > nbytes || (el->record && el->count > (nbytes - off) / el->record)) return "PLY file ended unexpectedly";
    *out = off;
    return nullptr;
  };
  const Element* vertex = nullptr;
  const Element* chunk = nullptr;
  const Element* sh = nullptr;
  for (const Element& e : elements) {
    if (e.name == "vertex" && !vertex) vertex = &e;
    if (e.name == "chunk" && !chunk) chunk = &e;
    if (e.name == "sh" && !sh) sh = &e;
  }
  if (!vertex) return "PLY has no vertex element";
  // splat indices are 32-bit on the device (as in SPZ files)
  if (vertex->count > 0x7fffffffull) return "PLY vertex count above 2^31 - 1";
  for (const Element& e : elements)
    if (e.count > 0x7fffffffull) return "PLY element count above 2^31 - 1";
  d->count = vertex->count;
  d->record = vertex->record;
  uint64_t off = 0;
  const char* err;
  const char* packed_names[4] = {"packed_position", "packed_rotation", "packed_scale", "packed_color"};
  bool compressed = chunk != nullptr;
  for (int k = 0; k < 4 && compressed; k++) compressed = find(*vertex, packed_names[k]) != nullptr;
  if (compressed) {
    for (const Element* el : {chunk, vertex})
      for (const Prop& p : el->props)
        if (p.list) {
          g_error = "PLY " + el->name + " list properties are not supported";
          return g_error.c_str();
        }
    static const char* chunk_names[18] = {"min_x", "min_y", "min_z", "max_x", "max_y", "max_z",
                                          "min_scale_x", "min_scale_y", "min_scale_z", "max_scale_x", "max_scale_y", "max_scale_z",
                                          "min_r", "min_g", "min_b", "max_r", "max_g", "max_b"};
    std::string missing;
    for (int k = 0; k < 12; k++)
      if (!find(*chunk, chunk_names[k])) missing += (missing.empty() ? "" : ", ") + std::string(chunk_names[k]);
    if (!missing.empty()) {
      g_error = "PLY chunk lacks " + missing;
      return g_error.c_str();
    }
    const uint64_t chunks = (vertex->count + 255) / 256;
    if (chunk->count < chunks) {
      g_error = "PLY has " + std::to_string(chunk->count) + " chunks for " + std::to_string(vertex->count) + " splats";
      return g_error.c_str();
    }
    d->kind = kPlyCompressed;
    for (int k = 0; k < 18; k++) d->chunk_prop[k] = pp(find(*chunk, chunk_names[k]));
    for (int k = 0; k < 4; k++) {
      const Prop* p = find(*vertex, packed_names[k]);
      if (kTypeBytes[p->type] != 4) return "PLY packed words must be 32-bit";
      d->packed[k] = pp(p);
    }
    uint64_t coff = 0;
    if ((err = offset_of(chunk, &coff))) return err;
    d->chunk = (const unsigned char*)(uintptr_t)coff;
    d->chunk_record = chunk->record;
    int rest = 0;
    if (sh)
      while (find(*sh, "f_rest_" + std::to_string(rest))) rest++;
    d->sh_degree = (sh && sh->count >= vertex->count) ? shdeg(rest) : 0;
    if (sh && d->sh_degree > 0) {
      uint64_t soff = 0;
      if ((err = offset_of(sh, &soff))) return err;
      d->sh = (const unsigned char*)(uintptr_t)soff;
      d->sh_record = sh->record;
      const int per = rest / 3;
      const int vals = (d->sh_degree == 1 ? 3 : d->sh_degree == 2 ? 8 : d->sh_degree == 3 ? 15 : 24) * 3;
      for (int v = 0; v < vals; v++) {
        const Prop* p = find(*sh, "f_rest_" + std::to_string((v % 3) * per + v / 3));
        d->sh_byte[v] = p ? p->offset : 0;
      }
    }
  } else {
    static const char* standard[14] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3",
                                       "opacity", "f_dc_0", "f_dc_1", "f_dc_2"};
    static const char* cloud[6] = {"x", "y", "z", "red", "green", "blue"};
    bool is_standard = true, is_cloud = true, any_standard = false;
    for (const char* n : standard) {
      const bool h = find(*vertex, n) != nullptr;
      is_standard = is_standard && h;
      any_standard = any_standard || h;
    }
    for (const char* n : cloud) is_cloud = is_cloud && find(*vertex, n) != nullptr;
    if (!is_standard && !is_cloud) {
      std::string missing;
      if (any_standard) {
        for (const char* n : standard)
          if (!find(*vertex, n)) missing += (missing.empty() ? "" : ", ") + std::string(n);
      } else {
        for (const char* n : cloud)
          if (!find(*vertex, n)) missing += (missing.empty() ? "" : ", ") + std::string(n);
      }
      g_error = "PLY vertex lacks " + missing;
      return g_error.c_str();
    }
    for (const Prop& p : vertex->props)
      if (p.list) return "PLY vertex list properties are not supported";
    d->kind = is_standard ? kPlyStandard : kPlyPoints;
    for (int k = 0; k < 3; k++) d->xyz[k] = pp(find(*vertex, standard[k]));
    if (is_standard) {
      for (int k = 0; k < 3; k++) d->scale[k] = pp(find(*vertex, standard[3 + k]));
      for (int k = 0; k < 4; k++) d->rot[k] = pp(find(*vertex, standard[6 + k]));
      d->opacity = pp(find(*vertex, "opacity"));
      for (int k = 0; k < 3; k++) d->color[k] = pp(find(*vertex, standard[11 + k]));
      int rest = 0;
      while (find(*vertex, "f_rest_" + std::to_string(rest))) rest++;
      d->sh_degree = shdeg(rest);
      const int per = rest / 3;
      const int vals = (d->sh_degree == 0 ? 0 : d->sh_degree == 1 ? 3 : d->sh_degree == 2 ? 8 : d->sh_degree == 3 ? 15 : 24) * 3;
      for (int v = 0; v < vals; v++) d->rest[v] = pp(find(*vertex, "f_rest_" + std::to_string((v % 3) * per + v / 3)));
    } else {
      for (int k = 0; k < 3; k++) d->color[k] = pp(find(*vertex, cloud[3 + k]));
      d->alpha = pp(find(*vertex, "alpha"));
      d->sh_degree = 0;
    }
  }
  if ((err = offset_of(vertex, &off))) return err;
  d->vertex = (const unsigned char*)(uintptr_t)off;
  d->out_degree = d->sh_degree;
  return nullptr;
}

cudaError_t launch_decode_ply(const PlyDesc& desc, float* centers, float* log_scales, float* quats, float* opacities,
                              float* colors, cudaStream_t stream) {
  if (desc.count == 0) return cudaSuccess;
  // standard files and point clouds: records staged a warp at a time
  if (desc.kind != kPlyCompressed && desc.record <= kRowsMaxRecord) {
    switch (desc.out_degree) {
      case 0: return launch_rows<3>(desc, centers, log_scales, quats, opacities, colors, stream);
      case 1: return launch_rows<12>(desc, centers, log_scales, quats, opacities, colors, stream);
      case 2: return launch_rows<27>(desc, centers, log_scales, quats, opacities, colors, stream);
      case 3: return launch_rows<48>(desc, centers, log_scales, quats, opacities, colors, stream);
      default: return launch_rows<75>(desc, centers, log_scales, quats, opacities, colors, stream);
    }
  }
  const uint32_t threads = 128;
  const uint64_t blocks = (desc.count + threads - 1) / threads;
  k_decode_ply<<<(unsigned)blocks, threads, 0, stream>>>(desc, centers, log_scales, quats, opacities, colors);
  return cudaGetLastError();
}

}  // namespace rdx
