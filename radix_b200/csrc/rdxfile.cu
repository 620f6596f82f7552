// RDX files (src/core/rdx.ts): the serialized bundles of an ArrayData in
// chunks of rows. Every piece is a container - u32 magic, u32 metaLength,
// u32 payloadCount, u32 0, JSON meta, u32 payloadSize[payloadCount], the
// payloads, each section 16-byte aligned. The header piece ("RDXH") names the
// bundles, their channels and formats, in payload order; each chunk ("RDXC")
// holds { start, count } and, per channel, that channel's elements gzipped
// with their bytes transposed (byte b of every element together).
//
// The host parses the JSON and inflates the payloads (DEFLATE is sequential
// within a stream, but every payload is a stream of its own, so host threads
// share them); the device transposes the bytes back, every chunk and channel
// in one launch, into the caller's channel arrays.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "rdx_internal.h"

namespace rdx {
namespace {

constexpr uint32_t kHeaderMagic = 0x48584452u;  // "RDXH"
constexpr uint32_t kChunkMagic = 0x43584452u;   // "RDXC"
constexpr int kRdxVersion = 1;

thread_local char g_error[256];  // the last error text of this thread

const char* error_text(const char* fmt, const char* a = "", const char* b = "", uint64_t x = 0, uint64_t y = 0) {
  snprintf(g_error, sizeof(g_error), fmt, a, b, (unsigned long long)x, (unsigned long long)y);
  return g_error;
}

uint32_t le32(const unsigned char* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
uint64_t align16(uint64_t n) { return (n + 15) & ~(uint64_t)15; }

// ---- a small JSON reader: objects keep their key order ----

struct Json {
  enum Kind { kNull, kBool, kNum, kStr, kArr, kObj } kind = kNull;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;
  const Json* get(const char* key) const {
    if (kind != kObj) return nullptr;
    for (const auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

struct JsonReader {
  const char* p;
  const char* end;
  int depth = 0;
  void ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  bool lit(const char* s) {
    const size_t n = strlen(s);
    if ((size_t)(end - p) < n || memcmp(p, s, n) != 0) return false;
    p += n;
    return true;
  }
  static void utf8(std::string& out, uint32_t c) {
    if (c < 0x80) {
      out += (char)c;
    } else if (c < 0x800) {
      out += (char)(0xC0 | (c >> 6));
      out += (char)(0x80 | (c & 0x3F));
    } else if (c < 0x10000) {
      out += (char)(0xE0 | (c >> 12));
      out += (char)(0x80 | ((c >> 6) & 0x3F));
      out += (char)(0x80 | (c & 0x3F));
    } else {
      out += (char)(0xF0 | (c >> 18));
      out += (char)(0x80 | ((c >> 12) & 0x3F));
      out += (char)(0x80 | ((c >> 6) & 0x3F));
      out += (char)(0x80 | (c & 0x3F));
    }
  }
  bool hex4(uint32_t* v) {
    if (end - p < 4) return false;
    *v = 0;
    for (int i = 0; i < 4; i++) {
      const char c = *p++;
      *v <<= 4;
      if (c >= '0' && c <= '9') *v |= (uint32_t)(c - '0');
      else if (c >= 'a' && c <= 'f') *v |= (uint32_t)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') *v |= (uint32_t)(c - 'A' + 10);
      else return false;
    }
    return true;
  }
  bool string(std::string& out) {
    if (p >= end || *p != '"') return false;
    p++;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        if (++p >= end) return false;
        const char e = *p++;
        switch (e) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            uint32_t c;
            if (!hex4(&c)) return false;
            if (c >= 0xD800 && c < 0xDC00 && end - p >= 6 && p[0] == '\\' && p[1] == 'u') {
              p += 2;
              uint32_t lo;
              if (!hex4(&lo)) return false;
              c = 0x10000 + ((c - 0xD800) << 10) + (lo - 0xDC00);
            }
            utf8(out, c);
            break;
          }
          default: return false;
        }
      } else {
        out += *p++;
      }
    }
    if (p >= end) return false;
    p++;
    return true;
  }
  bool value(Json& v) {
    if (++depth > 64) return false;
    ws();
    if (p >= end) return false;
    bool ok = true;
    if (*p == '{') {
      p++;
      v.kind = Json::kObj;
      ws();
      if (p < end && *p == '}') {
        p++;
      } else {
        while (ok) {
          ws();
          std::string key;
          if (!string(key)) return false;
          ws();
          if (p >= end || *p++ != ':') return false;
          v.obj.emplace_back(std::move(key), Json());
          if (!value(v.obj.back().second)) return false;
          ws();
          if (p < end && *p == ',') {
            p++;
            continue;
          }
          if (p < end && *p == '}') {
            p++;
            break;
          }
          return false;
        }
      }
    } else if (*p == '[') {
      p++;
      v.kind = Json::kArr;
      ws();
      if (p < end && *p == ']') {
        p++;
      } else {
        while (true) {
          v.arr.emplace_back();
          if (!value(v.arr.back())) return false;
          ws();
          if (p < end && *p == ',') {
            p++;
            continue;
          }
          if (p < end && *p == ']') {
            p++;
            break;
          }
          return false;
        }
      }
    } else if (*p == '"') {
      v.kind = Json::kStr;
      ok = string(v.str);
    } else if (lit("true")) {
      v.kind = Json::kBool;
      v.b = true;
    } else if (lit("false")) {
      v.kind = Json::kBool;
    } else if (lit("null")) {
      v.kind = Json::kNull;
    } else {
      char* stop = nullptr;
      std::string tok(p, (size_t)std::min<ptrdiff_t>(end - p, 64));
      v.num = strtod(tok.c_str(), &stop);
      if (stop == tok.c_str()) return false;
      v.kind = Json::kNum;
      p += stop - tok.c_str();
    }
    depth--;
    return ok;
  }
};

bool parse_json(const unsigned char* s, uint64_t n, Json* out) {
  JsonReader r{reinterpret_cast<const char*>(s), reinterpret_cast<const char*>(s) + n};
  if (!r.value(*out)) return false;
  r.ws();
  return r.p == r.end;
}

// Bytes of one element of an ArrayFormats name ("uint32x4", "float16", ...): 0 if invalid
int element_bytes(const std::string& f) {
  static const std::pair<const char*, int> kScalars[] = {{"uint8", 1},  {"sint8", 1},  {"unorm8", 1},  {"snorm8", 1},
                                                         {"uint16", 2}, {"sint16", 2}, {"float16", 2}, {"uint32", 4},
                                                         {"sint32", 4}, {"float32", 4}};
  const size_t x = f.find('x');
  const std::string scalar = f.substr(0, x);
  int components = 1;
  if (x != std::string::npos) {
    const std::string c = f.substr(x + 1);
    if (c.empty() || c.size() > 6 || c.find_first_not_of("0123456789") != std::string::npos) return 0;
    components = atoi(c.c_str());
    if (components < 1) return 0;
  }
  for (const auto& s : kScalars)
    if (scalar == s.first) return s.second * components;
  return 0;
}

// A container: its meta JSON and payload spans (offsets into `bytes`)
const char* read_container(const unsigned char* bytes, uint64_t n, uint32_t magic, Json* meta,
                           std::vector<std::pair<uint64_t, uint64_t>>* payloads, uint64_t* length) {
  if (n < 16 || le32(bytes) != magic) return "Not an RDX piece of the expected type";
  const uint64_t meta_len = le32(bytes + 4), count = le32(bytes + 8);
  const uint64_t sizes_at = 16 + align16(meta_len);
  if (16 + meta_len > n || sizes_at + count * 4 > n) return "RDX file ended unexpectedly";
  if (!parse_json(bytes + 16, meta_len, meta)) return "RDX piece with malformed JSON meta";
  uint64_t at = sizes_at + align16(count * 4);
  payloads->clear();
  for (uint64_t i = 0; i < count; i++) {
    const uint64_t size = le32(bytes + sizes_at + i * 4);
    if (at + size > n) return "RDX file ended unexpectedly";
    payloads->emplace_back(at, size);
    at += align16(size);
  }
  *length = at;
  return nullptr;
}

// A JSON number as a count: false unless it is a whole number in [0, 2^53)
// (the integers a JavaScript writer represents exactly)
bool as_u64(const Json* v, uint64_t* out) {
  *out = 0;
  if (!v || v->kind != Json::kNum || !(v->num >= 0.0) || v->num >= 9007199254740992.0) return false;
  if (v->num != (double)(uint64_t)v->num) return false;
  *out = (uint64_t)v->num;
  return true;
}

// Elements a chunk may hold (the reference's element indices are u32)
constexpr uint64_t kMaxChunkElements = 0xffffffffull;
// DEFLATE expands at most 1032:1, so a payload of n bytes inflates to fewer
// than this: larger claims are rejected before any buffer is sized by them
uint64_t max_inflated(uint64_t n) { return n * 1032 + 1024; }

// Inflate one gzip payload completely: the bytes, or -1 on a bad stream;
// stops (returning more than cap) once the output passes cap bytes
int64_t gunzip_all(const unsigned char* in, uint64_t n, std::vector<unsigned char>* out, uint64_t cap) {
  z_stream zs;
  memset(&zs, 0, sizeof(zs));
  if (inflateInit2(&zs, 16 + MAX_WBITS) != Z_OK) return -1;
  out->clear();
  unsigned char buf[1 << 16];
  zs.next_in = const_cast<unsigned char*>(in);
  zs.avail_in = (uInt)n;
  int status = Z_OK;
  while (status == Z_OK) {
    zs.next_out = buf;
    zs.avail_out = sizeof(buf);
    status = inflate(&zs, Z_NO_FLUSH);
    if (status != Z_OK && status != Z_STREAM_END) break;
    out->insert(out->end(), buf, buf + (sizeof(buf) - zs.avail_out));
    if (out->size() > cap) break;  // more than the chunk claims: a size mismatch, not a bad stream
    if (status == Z_OK && zs.avail_in == 0 && zs.avail_out != 0) {
      status = Z_BUF_ERROR;
      break;
    }
  }
  inflateEnd(&zs);
  if (out->size() > cap) return (int64_t)out->size();
  return status == Z_STREAM_END ? (int64_t)out->size() : -1;
}

// ---- device: bytes transposed back ----

constexpr int kTransposeThreads = 256;

// A piece of 16-byte elements whose rows come in fours and whose byte planes
// are word-aligned (its source) and whose elements are 16-byte aligned (its
// destination) goes four elements a thread
__host__ __device__ __forceinline__ bool by_quads(const RdxPiece& pc, const unsigned char* staged) {
  return pc.bytes == 16 && pc.count % 4 == 0 && ((uintptr_t)(staged + pc.src) & 3u) == 0 &&
         ((uintptr_t)pc.dst & 15u) == 0;
}

// Element i's byte b sits at src[b * count + i]: blockIdx.y picks the piece
__global__ void __launch_bounds__(kTransposeThreads) k_untranspose(const RdxPiece* __restrict__ pieces,
                                                                   const unsigned char* __restrict__ staged) {
  const RdxPiece pc = pieces[blockIdx.y];
  const unsigned char* src = staged + pc.src;
  if (by_quads(pc, staged)) {
    // one word of each of the 16 byte planes (elements 4g to 4g + 3), then a
    // 4x4 byte transpose for each of the elements' four words
    const uint32_t* planes = reinterpret_cast<const uint32_t*>(src);
    const uint32_t quads = pc.count / 4;
    uint4* dst = reinterpret_cast<uint4*>(pc.dst);
    for (uint32_t g = blockIdx.x * kTransposeThreads + threadIdx.x; g < quads; g += gridDim.x * kTransposeThreads) {
      uint32_t p[16];
#pragma unroll
      for (int b = 0; b < 16; b++) p[b] = __ldg(planes + (uint64_t)b * quads + g);
      uint32_t e[4][4];  // e[j][k]: word k of element 4g + j (bytes 4k to 4k + 3: planes 4k to 4k + 3, byte j)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t lo01 = __byte_perm(p[4 * k], p[4 * k + 1], 0x5140), lo23 = __byte_perm(p[4 * k + 2], p[4 * k + 3], 0x5140);
        const uint32_t hi01 = __byte_perm(p[4 * k], p[4 * k + 1], 0x7362), hi23 = __byte_perm(p[4 * k + 2], p[4 * k + 3], 0x7362);
        e[0][k] = __byte_perm(lo01, lo23, 0x5410);
        e[1][k] = __byte_perm(lo01, lo23, 0x7632);
        e[2][k] = __byte_perm(hi01, hi23, 0x5410);
        e[3][k] = __byte_perm(hi01, hi23, 0x7632);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) dst[(uint64_t)g * 4 + j] = make_uint4(e[j][0], e[j][1], e[j][2], e[j][3]);
    }
    return;
  }
  for (uint32_t i = blockIdx.x * kTransposeThreads + threadIdx.x; i < pc.count; i += gridDim.x * kTransposeThreads) {
    unsigned char* d = pc.dst + (uint64_t)i * pc.bytes;
    if (pc.bytes == 16 && (reinterpret_cast<uintptr_t>(d) & 15u) == 0) {
      uint32_t w[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        w[k] = (uint32_t)src[(uint64_t)(4 * k) * pc.count + i] | ((uint32_t)src[(uint64_t)(4 * k + 1) * pc.count + i] << 8) |
               ((uint32_t)src[(uint64_t)(4 * k + 2) * pc.count + i] << 16) |
               ((uint32_t)src[(uint64_t)(4 * k + 3) * pc.count + i] << 24);
      }
      *reinterpret_cast<uint4*>(d) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
      for (uint32_t b = 0; b < pc.bytes; b++) d[b] = src[(uint64_t)b * pc.count + i];
    }
  }
}

}  // namespace

const char* rdxfile_header(const unsigned char* bytes, uint64_t nbytes, RdxFile* f) {
  *f = RdxFile();
  if (!bytes || nbytes < 16 || le32(bytes) != kHeaderMagic) return "Not an RDX piece of the expected type";
  Json meta;
  std::vector<std::pair<uint64_t, uint64_t>> payloads;
  uint64_t length = 0;
  const char* err = read_container(bytes, nbytes, kHeaderMagic, &meta, &payloads, &length);
  if (err) return err;
  f->header_bytes = length;
  f->header_json.assign(reinterpret_cast<const char*>(bytes) + 16, le32(bytes + 4));
  const Json* version = meta.get("version");
  if (!version || version->kind != Json::kNum || version->num != kRdxVersion)
    return error_text("RDX version %s is not 1", version && version->kind == Json::kNum ? std::to_string((long long)version->num).c_str() : "undefined");
  if (!as_u64(meta.get("count"), &f->count)) return "RDX header without a valid count";
  if (f->count > kMaxChunkElements) return error_text("RDX header count %s%s%llu is above 2^32 - 1", "", "", f->count);
  if (meta.get("chunkSize") && !as_u64(meta.get("chunkSize"), &f->chunk_size)) return "RDX header with an invalid chunkSize";
  const Json* bundles = meta.get("bundles");
  if (!bundles || bundles->kind != Json::kObj) return "RDX header without bundles";
  for (const auto& b : bundles->obj) {
    const Json* def = b.second.get("def");
    const Json* channels = def ? def->get("channels") : nullptr;
    if (!channels || channels->kind != Json::kObj) return error_text("RDX bundle %s without channels", b.first.c_str());
    for (const auto& c : channels->obj) {
      if (c.second.kind != Json::kStr) return error_text("RDX channel %s.%s without a format", b.first.c_str(), c.first.c_str());
      const int eb = element_bytes(c.second.str);
      if (eb == 0) return error_text("Invalid array format \"%s\"", c.second.str.c_str());
      f->channels.push_back({b.first, c.first, c.second.str, eb});
    }
  }
  const Json* chunks = meta.get("chunks");
  if (!chunks || chunks->kind != Json::kArr) return "RDX header without chunks";
  uint64_t total = length;
  for (const Json& c : chunks->arr) {
    uint64_t b = 0;
    if (!as_u64(&c, &b)) return "RDX header with an invalid chunk size";
    if (b > nbytes - std::min(total, nbytes)) return "RDX file ended unexpectedly";
    f->chunk_bytes.push_back(b);
    total += b;
  }
  if (total > nbytes) return "RDX file ended unexpectedly";
  return nullptr;
}

void parallel_for(size_t n, uint64_t work_bytes, const std::function<void(size_t)>& fn) {
  // a thread per MB of input at most, up to the host's threads (32 at most)
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t threads = (size_t)std::min<uint64_t>({(uint64_t)hw, (uint64_t)n, 32, 1 + work_bytes / (1u << 20)});
  std::atomic<size_t> next{0};
  auto drain = [&] {
    for (size_t i = next++; i < n; i = next++) fn(i);
  };
  std::vector<std::thread> pool;
  for (size_t t = 1; t < threads; t++) {
    try {
      pool.emplace_back(drain);
    } catch (...) {
      break;  // no more threads: the others and this one share the rest
    }
  }
  drain();
  for (auto& th : pool) th.join();
}

const char* rdxfile_unpack(const unsigned char* bytes, uint64_t nbytes, const RdxFile& f, const bool* wanted,
                           std::vector<unsigned char>* staged, std::vector<RdxSpan>* spans) {
  (void)nbytes;  // rdxfile_header checked that every chunk lies inside the file
  staged->clear();
  spans->clear();
  // Every chunk's container first (in file order, stopping at the first bad
  // one), then every payload inflated, the payloads shared among host threads
  // (each is its own gzip stream); errors are reported in the order a serial
  // read would meet them
  struct Payload {
    const unsigned char* in;
    uint64_t size, expect, start, dst;
    int channel;
    bool keep;
  };
  std::vector<Payload> jobs;
  const char* parse_error = nullptr;
  uint64_t at = f.header_bytes, total = 0, packed = 0;
  for (size_t ci = 0; ci < f.chunk_bytes.size() && !parse_error; ci++) {
    Json meta;
    std::vector<std::pair<uint64_t, uint64_t>> payloads;
    uint64_t length = 0;
    const char* err = read_container(bytes + at, f.chunk_bytes[ci], kChunkMagic, &meta, &payloads, &length);
    uint64_t start = 0, count = 0;
    if (err) {
      parse_error = err;
    } else if (!as_u64(meta.get("start"), &start) || !as_u64(meta.get("count"), &count)) {
      parse_error = error_text("RDX chunk %s%s%llu without a valid start and count", "", "", (uint64_t)ci);
    } else if (count > kMaxChunkElements) {
      parse_error = error_text("RDX chunk %s%s%llu holds %llu elements (at most 2^32 - 1)", "", "", (uint64_t)ci, count);
    } else if (start > f.count || count > f.count - start) {
      parse_error = error_text("RDX chunk at %s%s%llu runs past the %llu elements", "", "", start, f.count);
    } else if (payloads.size() != f.channels.size()) {
      parse_error = error_text("RDX chunk %s%s%llu holds %llu payloads", "", "", (uint64_t)ci, (uint64_t)payloads.size());
    } else {
      for (size_t k = 0; k < f.channels.size() && !parse_error; k++) {
        const uint64_t eb = (uint64_t)f.channels[k].element_bytes;
        if (count * eb > max_inflated(payloads[k].second)) {
          // more bytes than the payload can inflate to: refused before any buffer is sized by it
          const RdxChannel& ch = f.channels[k];
          parse_error = error_text("Chunk at %s: %s expects %llu bytes from a %llu-byte payload",
                                   std::to_string(start).c_str(), (ch.bundle + "." + ch.label).c_str(), count * eb,
                                   payloads[k].second);
          break;
        }
        Payload j{bytes + at + payloads[k].first, payloads[k].second, count * eb, start, total, (int)k,
                  wanted[k] && count > 0};
        if (j.keep) {
          spans->push_back({total, (int)k, start, (uint32_t)count, (uint32_t)eb});
          total += j.expect;
        }
        packed += j.size;
        jobs.push_back(j);
      }
    }
    at += f.chunk_bytes[ci];
  }
  try {
    staged->resize(total);
  } catch (const std::exception&) {
    return error_text("RDX file needs %s%s%llu bytes of host memory to inflate", "", "", total);
  }
  constexpr int64_t kNoMemory = -2;
  std::vector<int64_t> got(jobs.size(), 0);
  parallel_for(jobs.size(), packed, [&](size_t q) {
    const Payload& j = jobs[q];
    try {
      std::vector<unsigned char> buf;
      buf.reserve(j.expect);
      got[q] = gunzip_all(j.in, j.size, &buf, j.expect);
      if (j.keep && got[q] == (int64_t)j.expect) memcpy(staged->data() + j.dst, buf.data(), buf.size());
    } catch (const std::exception&) {
      got[q] = kNoMemory;  // no exception leaves a worker thread
    }
  });
  for (size_t q = 0; q < jobs.size(); q++) {
    const Payload& j = jobs[q];
    if (got[q] == kNoMemory) return "RDX payload could not be inflated: out of host memory";
    if (got[q] < 0) return "RDX payload is not a gzip stream";
    if ((uint64_t)got[q] != j.expect) {
      const RdxChannel& ch = f.channels[j.channel];
      return error_text("Chunk at %s: %s holds %llu bytes, expected %llu", std::to_string(j.start).c_str(),
                        (ch.bundle + "." + ch.label).c_str(), (uint64_t)got[q], j.expect);
    }
  }
  if (parse_error) spans->clear();
  return parse_error;
}

cudaError_t launch_untranspose(const RdxPiece* pieces_dev, const RdxPiece* pieces_host, int n_pieces,
                               const unsigned char* staged,
                               cudaStream_t stream) {
  // threads' work: a quarter of the rows for pieces taken four elements a thread
  uint32_t max_work = 0;
  for (int k = 0; k < n_pieces; k++)
    max_work = std::max(max_work, by_quads(pieces_host[k], staged) ? pieces_host[k].count / 4 : pieces_host[k].count);
  if (max_work == 0) return cudaSuccess;
  const uint32_t gx = std::min<uint32_t>((max_work + kTransposeThreads - 1) / kTransposeThreads, 1024u);
  for (int first = 0; first < n_pieces; first += 65535) {
    const int batch = std::min(n_pieces - first, 65535);
    k_untranspose<<<dim3(gx, (unsigned)batch), kTransposeThreads, 0, stream>>>(pieces_dev + first, staged);
  }
  return cudaGetLastError();
}

}  // namespace rdx
