"""Writers of RDX test files (src/core/rdx.ts:42-155, restated): bundles of
channels serialized in chunks of rows; every piece a container (u32 magic,
u32 meta length, u32 payload count, u32 0, JSON meta, u32 payload sizes,
payloads; sections 16-byte aligned), each payload one chunk of one channel
with its bytes transposed and gzipped."""
import gzip
import json
import struct

import numpy as np

HEADER_MAGIC = 0x48584452  # "RDXH"
CHUNK_MAGIC = 0x43584452   # "RDXC"
SCALAR_BYTES = {"uint8": 1, "sint8": 1, "unorm8": 1, "snorm8": 1, "uint16": 2, "sint16": 2, "float16": 2,
                "uint32": 4, "sint32": 4, "float32": 4}


def element_bytes(fmt):
    scalar, _, count = fmt.partition("x")
    return SCALAR_BYTES[scalar] * (int(count) if count else 1)


def _align16(n):
    return (n + 15) // 16 * 16


def container(magic, meta, payloads):
    text = json.dumps(meta, separators=(",", ":")).encode()
    sizes_at = 16 + _align16(len(text))
    payloads_at = sizes_at + _align16(4 * len(payloads))
    out = bytearray(payloads_at + sum(_align16(len(p)) for p in payloads))
    struct.pack_into("<IIII", out, 0, magic, len(text), len(payloads), 0)
    out[16:16 + len(text)] = text
    at = payloads_at
    for i, p in enumerate(payloads):
        struct.pack_into("<I", out, sizes_at + 4 * i, len(p))
        out[at:at + len(p)] = p
        at += _align16(len(p))
    return bytes(out)


def transposed_gzip(raw, eb, level=9):
    """Byte k of every element together, then gzip (Compression.compressTransposed)."""
    a = np.frombuffer(raw, dtype=np.uint8).reshape(-1, eb)
    return gzip.compress(np.ascontiguousarray(a.T).tobytes(), compresslevel=level, mtime=0)


def rdx_file(bundles, count, chunk_size=65536, meta=None, level=9):
    """A whole RDX file. bundles: {name: (channels {label: format}, bundle meta, {label: numpy array [count, ...]})},
    in payload order; payloads gzipped at `level`."""
    assert chunk_size > 0 and chunk_size % 4096 == 0
    chunks = []
    for start in range(0, count, chunk_size):
        n = min(chunk_size, count - start)
        payloads = []
        for channels, _, data in bundles.values():
            for label, fmt in channels.items():
                eb = element_bytes(fmt)
                raw = np.ascontiguousarray(data[label]).view(np.uint8).reshape(count, -1)
                assert raw.shape[1] == eb, (label, raw.shape, eb)
                payloads.append(transposed_gzip(raw[start:start + n].tobytes(), eb, level))
        chunks.append(container(CHUNK_MAGIC, {"start": start, "count": n}, payloads))
    header = {"version": 1, "count": count, "chunkSize": chunk_size, "meta": meta or {},
              "bundles": {name: {"def": {"channels": channels, "packing": "float32", "serialize": True},
                                 "meta": bmeta} for name, (channels, bmeta, _) in bundles.items()},
              "chunks": [len(c) for c in chunks]}
    return container(HEADER_MAGIC, header, []) + b"".join(chunks)
