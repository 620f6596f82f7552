"""radix_b200: the per-frame splat path of @sparkjsdev/radix on B200 (sm_100a).

Host-side mirror of the reference's interfaces for this path, over the C ABI
(include/radix_b200.h, radix_b200/lib/libradix_b200.so):

  SortKeys        src/core/sort.ts            compute / sort / invalid / validMax
  RadixSort       src/wgpu/WgpuRadixSort.ts   sort / sort_indirect (key-value, in place)
  Compact         src/wgpu/WgpuCompact.ts     order-preserving compaction
  SplatSorter     src/wgpu/WgpuSplatSorter.ts compact + sort + draw arguments
  project_collection  src/render/SplatProjector.ts:106-139 (ewa, fused with SH and keys)
  frame           project + sort, as SplatRenderer.update runs them

Arrays are torch tensors (CUDA or CPU) or numpy arrays. Every computation
runs in the CUDA library; there is no CPU fallback, and a missing build
raises.
"""
import ctypes
from dataclasses import dataclass, fields

import numpy as np

from . import _abi
from ._abi import RadixError
from .camera import IDENTITY, Camera, look_at, perspective

__all__ = [
    "Context", "SortKeys", "RadixSort", "Compact", "SplatSorter", "SplatParams", "Table", "SplatObject",
    "Camera", "look_at", "perspective", "project_collection", "project_backward", "frame", "frame_batched", "Batch",
    "RadixError", "decode_ply", "ply_info", "decode_spz", "spz_info", "rdxfile_info", "decode_rdxfile",
    "rdxfile_table",
    "align_capacity",
]

ROW_ELEMENTS = 4096  # TextureLayout.ROW_ELEMENTS (src/core/layout.ts:28-30)


def align_capacity(count):
    """TextureLayout.alignCapacity (src/core/layout.ts:70-72): whole 4096-element rows, at least one."""
    return max(1, -(-int(count) // ROW_ELEMENTS)) * ROW_ELEMENTS


def _torch():
    import torch
    return torch


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _ptr(x):
    if x is None:
        return None
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("radix_b200: tensors must be contiguous")
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("radix_b200: arrays must be C-contiguous")
        return x.ctypes.data
    raise TypeError(f"radix_b200: expected a torch tensor or numpy array, got {type(x)}")


def _on_cuda(x):
    return _is_torch(x) and x.is_cuda


def _empty_like_place(ref, shape, dtype_np):
    """An output array where `ref` lives: CUDA tensor for a CUDA input, else numpy."""
    if _on_cuda(ref):
        torch = _torch()
        tdt = {np.uint32: torch.int32, np.float32: torch.float32}[dtype_np]
        return torch.empty(shape, dtype=tdt, device=ref.device)
    return np.empty(shape, dtype=dtype_np)


class Context:
    """A device context (rdx_ctx): stream, scratch and error state. Calls run
    on torch's current stream of the context's device."""

    def __init__(self, device=0):
        self.device = device
        h = ctypes.c_void_p()
        st = _abi.lib().rdx_ctx_create(device, ctypes.byref(h))
        if st != _abi.RDX_OK:
            raise RadixError(st, f"radix_b200: no CUDA device {device} (rdx_ctx_create status {st})")
        self.handle = h

    def _bind_stream(self):
        try:
            torch = _torch()
            if torch.cuda.is_available():
                h = torch.cuda.current_stream(self.device).cuda_stream
                # torch's default stream is the legacy default stream: handle 0 there,
                # cudaStreamLegacy (0x1) for the C ABI, where NULL means the context's own
                _abi.lib().rdx_ctx_set_stream(self.handle, ctypes.c_void_p(h if h else 0x1))
        except ImportError:
            pass

    def call(self, name, *args):
        self._bind_stream()
        _abi.check(getattr(_abi.lib(), name)(self.handle, *args), self.handle)

    def synchronize(self):
        _abi.check(_abi.lib().rdx_ctx_synchronize(self.handle), self.handle)

    def set_profiling(self, on=True):
        """Record CUDA events around each phase (project, sort, copies) of later calls."""
        _abi.check(_abi.lib().rdx_ctx_set_profiling(self.handle, 1 if on else 0), self.handle)

    def set_wait(self, polls=0, silent_pass=-1):
        """Polls of a bounded device wait before it gives up (0: the default), and
        the test hook that silences the first tile of one digit pass of the next sort."""
        _abi.check(_abi.lib().rdx_ctx_set_wait(self.handle, int(polls), int(silent_pass)), self.handle)

    def set_sort_variant(self, variant=-1):
        """How sorts run their digit passes: -1 tuned for the shape or 0; 0
        onesweep kernels with tiles by size; 1-3 one cooperative kernel
        (1024x16, 512x16, 1024x8 threads x keys); 4-6 onesweep kernels with
        4096-, 2048- or 1024-key tiles."""
        _abi.check(_abi.lib().rdx_ctx_set_sort_variant(self.handle, int(variant)), self.handle)

    def tune_sort(self, keys, count, bits, reps=5):
        """Time every digit-pass variant on `count` device keys and remember the
        fastest for sorts of that shape; returns the timings."""
        r = _abi.rdx_tune_result()
        self.call("rdx_sort_tune", _ptr(keys), int(count), int(bits), int(reps), ctypes.byref(r))
        return r.as_dict()

    def phase_times(self):
        """{phase: (summed ms, runs)} since the last read (waits for the stream)."""
        ms = (ctypes.c_double * _abi.RDX_PHASES)()
        runs = (ctypes.c_uint64 * _abi.RDX_PHASES)()
        _abi.check(_abi.lib().rdx_ctx_phase_times(self.handle, ms, runs), self.handle)
        names = ("project", "sort", "copy_in", "copy_out", "batch")
        return {names[i]: (ms[i], runs[i]) for i in range(_abi.RDX_PHASES)}

    def launches(self):
        """Kernels this context has launched."""
        n = ctypes.c_uint64(0)
        _abi.check(_abi.lib().rdx_ctx_launches(self.handle, ctypes.byref(n)), self.handle)
        return n.value

    def set_host_reads(self, in_place=True):
        """Host tables: read the drawn candidates' rows of pinned columns in
        place (True, the default), or copy every host column in (False)."""
        _abi.check(_abi.lib().rdx_ctx_set_host_reads(self.handle, 1 if in_place else 0), self.handle)

    def host_bytes(self):
        """Bytes of table columns moved from host memory since the last query
        (copies and rows read in place); waits for the context's stream."""
        n = ctypes.c_uint64(0)
        _abi.check(_abi.lib().rdx_ctx_host_bytes(self.handle, ctypes.byref(n)), self.handle)
        return n.value

    def reserve(self, max_keys):
        _abi.check(_abi.lib().rdx_ctx_reserve(self.handle, int(max_keys)), self.handle)

    def close(self):
        if getattr(self, "handle", None):
            _abi.lib().rdx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def default_context(device=0):
    if device not in _contexts:
        _contexts[device] = Context(device)
    return _contexts[device]


def _ctx(ctx, *arrays):
    if ctx is not None:
        return ctx
    for a in arrays:
        if _on_cuda(a):
            return default_context(a.device.index or 0)
    return default_context(0)


class SortKeys:
    """src/core/sort.ts:27-83. invalid / valid_max are integer constants of a
    width; compute and sort run on the GPU."""

    KEY16_LO = 95 << 23
    KEY16_HI = (159 << 23) - 1

    @staticmethod
    def invalid(bits):
        return 2 ** bits - 1

    @staticmethod
    def valid_max(bits):
        return 0xFF * 2 ** (bits - 8) - 1

    @staticmethod
    def compute(distances, bits, ctx=None):
        """Keys of float64 distances (SortKeys.compute), or of float32 ones
        (GpuSortKeys.compute: max(d, 0)); uint32 where the distances live."""
        dt = str(distances.dtype)
        n = int(np.prod(distances.shape))
        keys = _empty_like_place(distances, (n,), np.uint32)
        c = _ctx(ctx, distances)
        if "float64" in dt:
            c.call("rdx_sort_keys_compute", _ptr(distances), n, bits, _ptr(keys))
        elif "float32" in dt:
            c.call("rdx_sort_keys_compute_f32", _ptr(distances), n, bits, _ptr(keys))
        else:
            raise TypeError("SortKeys.compute: float64 or float32 distances")
        return keys

    @staticmethod
    def sort(keys, count=None, bits=32, ordering=None, ctx=None):
        """Stable ascending order of the first `count` keys into `ordering`
        (default: a new array of align_capacity(count)); returns (ordering, visible)."""
        count = int(np.prod(keys.shape)) if count is None else int(count)
        if ordering is None:
            ordering = _empty_like_place(keys, (align_capacity(count),), np.uint32)
            if isinstance(ordering, np.ndarray):
                ordering[:] = 0
            else:
                ordering.zero_()
        visible = ctypes.c_uint32(0)
        _ctx(ctx, keys).call("rdx_sort", _ptr(keys), count, bits, _ptr(ordering), int(np.prod(ordering.shape)),
                             ctypes.byref(visible))
        return ordering, visible.value


class RadixSort:
    """WgpuRadixSort (src/wgpu/WgpuRadixSort.ts:56-141): sorts the caller's
    keys and values in place, ascending and stable."""

    def __init__(self, keys, values, ctx=None):
        self.keys = keys
        self.values = values
        self.ctx = _ctx(ctx, keys)

    def sort(self, count, bits=32):
        if bits not in (16, 24, 32):
            raise ValueError(f"WgpuRadixSort: bits must be 16, 24 or 32 (got {bits})")
        if count <= 0:
            return
        self.ctx.call("rdx_sort_pairs", _ptr(self.keys), _ptr(self.values), int(count), bits)

    def sort_indirect(self, count_buffer, bits=32):
        """Sort the first min(count_buffer[0], capacity) pairs, the count read on the GPU."""
        cap = int(np.prod(self.keys.shape))
        self.ctx.call("rdx_sort_pairs_indirect", _ptr(self.keys), _ptr(self.values), _ptr(count_buffer), cap, bits)


class Compact:
    """WgpuCompact (src/wgpu/WgpuCompact.ts:22-132): the keys that are not
    `invalid`, with their indices, in input order, and their count."""

    def __init__(self, ctx=None, invalid=0xFFFFFFFF):
        self.ctx = ctx
        self.invalid = invalid

    def compact(self, keys, n=None):
        n = int(np.prod(keys.shape)) if n is None else int(n)
        c = _ctx(self.ctx, keys)
        out_k = _empty_like_place(keys, (max(n, 1),), np.uint32)
        out_v = _empty_like_place(keys, (max(n, 1),), np.uint32)
        count = _empty_like_place(keys, (1,), np.uint32)
        c.call("rdx_compact", _ptr(keys), n, ctypes.c_uint32(self.invalid), _ptr(out_k), _ptr(out_v), _ptr(count))
        return out_k, out_v, count


class SplatSorter:
    """WgpuSplatSorter (src/wgpu/WgpuSplatSorter.ts:19-84): compaction of the
    invalid keys, a back-to-front sort, and drawIndexedIndirect arguments."""

    QUADS_PER_INSTANCE = 1024

    def __init__(self, ctx=None):
        self.ctx = ctx
        self.values = None
        self.count = None
        self.indirect = None

    def sort(self, keys, count, bits):
        c = _ctx(self.ctx, keys)
        self.values = _empty_like_place(keys, (max(int(count), 1),), np.uint32)
        self.count = _empty_like_place(keys, (1,), np.uint32)
        self.indirect = _empty_like_place(keys, (5,), np.uint32)
        c.call("rdx_splat_sort", _ptr(keys), int(count), bits, _ptr(self.values), _ptr(self.count), _ptr(self.indirect))
        return self.values, self.count, self.indirect

    def read_count(self):
        return int(np.asarray(self.count.cpu() if _is_torch(self.count) else self.count)[0])


@dataclass
class SplatParams:
    """SplatViewParams + SplatObjectParams with the reference's defaults
    (src/render/splatParams.ts:68-72)."""

    max_std_dev: float = float(np.sqrt(8.0))
    min_alpha: float = 0.5 / 255
    falloff: float = 1.0
    lod_inflate: bool = True
    blur_amount: float = 0.3
    pre_blur_amount: float = 0.0
    clip_xy: float = 1.4
    min_pixel_radius: float = 0.0
    max_pixel_radius: float = 512.0
    min_contribution: float = 0.0
    focal_distance: float = 0.0
    aperture_tan: float = 0.0
    sort_guard: float = 0.0
    max_sh_degree: int = 4

    def to_c(self):
        p = _abi.rdx_params()
        for f in fields(self):
            v = getattr(self, f.name)
            setattr(p, f.name, int(v) if f.name in ("lod_inflate", "max_sh_degree") else float(v))
        return p


class Table:
    """A splat table (rdx_table): raw float32 columns or Radix's ext layout."""

    def __init__(self, c_table, keep):
        self.c = c_table
        self._keep = keep

    @property
    def count(self):
        return int(self.c.count)

    @classmethod
    def raw(cls, centers, log_scales, quats, opacities, colors, sh_degree=None):
        n = int(centers.shape[0])
        k = int(colors.shape[1]) - 1 if len(colors.shape) == 3 else int(colors.shape[1]) // 3 - 1
        deg = {0: 0, 3: 1, 8: 2, 15: 3, 24: 4}[k] if sh_degree is None else sh_degree
        t = _abi.rdx_table()
        t.layout = _abi.RDX_LAYOUT_RAW
        t.sh_degree = deg
        t.color_dtype = _abi.RDX_DTYPE_F16 if "float16" in str(colors.dtype) else _abi.RDX_DTYPE_F32
        t.count = n
        t.centers, t.log_scales, t.quats = _ptr(centers), _ptr(log_scales), _ptr(quats)
        t.opacities, t.colors = _ptr(opacities), _ptr(colors)
        return cls(t, [centers, log_scales, quats, opacities, colors])

    @staticmethod
    def _sh(t, keep, sh, sh_degree, sh_codec, palette):
        t.sh_degree = sh_degree
        t.sh_codec = _abi.RDX_SH_PACKED if sh_codec == "packed" else _abi.RDX_SH_EXT
        if palette is not None:
            entries, labels, stride = palette
            t.sh_palette, t.sh_label = _ptr(entries), _ptr(labels)
            t.sh_stride = int(stride)
            t.sh_palette_size = int(entries.shape[0]) // int(stride)
            keep += [entries, labels]
        for i, ch in enumerate(sh):
            t.ext_sh[i] = _ptr(ch)
        keep += list(sh)

    @classmethod
    def ext(cls, ext_a, ext_b, ext_sh=(), sh_degree=0, sh_codec="ext", palette=None):
        """extA / extB uint32x4 columns (src/core/splats.ts:10-24) and the SH
        texel channels of codec sh_codec ("ext" or "packed"), each [count][4]
        uint32, or palette = (entries [size * stride][4] uint32, labels [count]
        uint16, stride) (src/core/sh.ts:13-24, 432-527)."""
        t = _abi.rdx_table()
        t.layout = _abi.RDX_LAYOUT_EXT
        t.count = int(ext_a.shape[0])
        t.ext_a, t.ext_b = _ptr(ext_a), _ptr(ext_b)
        keep = [ext_a, ext_b]
        cls._sh(t, keep, ext_sh, sh_degree, sh_codec, palette)
        return cls(t, keep)

    @classmethod
    def cov(cls, cov_a, cov_b, sh=(), sh_degree=0, sh_codec="ext", palette=None):
        """covA / covB uint32x4 columns (src/core/splats.ts:25-27), SH as for ext."""
        t = _abi.rdx_table()
        t.layout = _abi.RDX_LAYOUT_COV
        t.count = int(cov_a.shape[0])
        t.ext_a, t.ext_b = _ptr(cov_a), _ptr(cov_b)
        keep = [cov_a, cov_b]
        cls._sh(t, keep, sh, sh_degree, sh_codec, palette)
        return cls(t, keep)

    PACKED_ENCODING = (0.0, 1.0, -12.0, 9.0)  # Splats.DEFAULT_PACKED_ENCODING (src/core/splats.ts:97)

    @classmethod
    def packed(cls, packed, encoding=PACKED_ENCODING, sh=(), sh_degree=0, sh_codec="ext", palette=None):
        """The packed uint32x4 column (src/core/splats.ts:28-32) and its
        encoding (rgbMin, rgbMax, lnScaleMin, lnScaleMax), SH as for ext."""
        t = _abi.rdx_table()
        t.layout = _abi.RDX_LAYOUT_PACKED
        t.count = int(packed.shape[0])
        t.packed = _ptr(packed)
        t.packed_encoding[:] = [float(x) for x in encoding]
        keep = [packed]
        cls._sh(t, keep, sh, sh_degree, sh_codec, palette)
        return cls(t, keep)

    @classmethod
    def from_dict(cls, d, to=None):
        """A raw table of a synthetic dict, its columns moved with `to(array)`."""
        f = to or (lambda a: a)
        return cls.raw(f(d["centers"]), f(d["log_scales"]), f(d["quats"]), f(d["opacities"]), f(d["colors"]),
                       d["sh_degree"])


class SplatObject:
    """One object of a collection: `count` splats of `table` drawn with
    `world` (column-major object -> world), optional per-object params."""

    def __init__(self, table, count=None, world=None, params=None):
        self.table = table
        self.count = table.count if count is None else int(count)
        self.world = IDENTITY if world is None else np.asarray(world, dtype=np.float64).reshape(16)
        self.params = params


def _c_objects(objects):
    arr = (_abi.rdx_object * max(1, len(objects)))()
    keep = []
    for i, o in enumerate(objects):
        arr[i].table = ctypes.pointer(o.table.c)
        arr[i].count = o.count
        arr[i].world[:] = list(o.world)
        if o.params is not None:
            p = o.params.to_c()
            keep.append(p)
            arr[i].params = ctypes.pointer(p)
        keep.append(o.table)
    return arr, keep


OUTPUT_SHAPES = {  # per eye: trailing shape, dtype
    "mean2d": ((2,), np.float32),
    "conic": ((3,), np.float32),
    "depth": ((), np.float32),
    "opacity": ((), np.float32),
    "rgb": ((3,), np.float32),
    "radii": ((3,), np.float32),
}


def _alloc_outputs(names, n, eyes, device):
    torch = _torch()
    out = {}
    for name in names:
        if name == "words":
            shape, dt = (n, 4 * eyes), torch.int32
        elif name == "keys":
            shape, dt = (n,), torch.int32
        else:
            tail, _ = OUTPUT_SHAPES[name]
            shape, dt = (eyes, n, *tail), torch.float32
        if device is None:
            out[name] = np.empty(shape, dtype=np.uint32 if dt is torch.int32 else np.float32)
        else:
            out[name] = torch.empty(shape, dtype=dt, device=device)
    return out


def _c_outputs(out):
    o = _abi.rdx_outputs()
    for name, arr in out.items():
        setattr(o, name, _ptr(arr))
    return o


DEFAULT_OUTPUTS = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")


def project_collection(objects, camera, params=None, sort_bits=24, pass_="full", cull_keys=False,
                       outputs=DEFAULT_OUTPUTS, device="cuda", ctx=None, out=None):
    """projectCollection with the ewa method: outputs (per eye [E][n][...],
    words [n][4E], keys [n]) as CUDA tensors (device=None: numpy), or into
    `out` (a dict of such arrays) when given."""
    params = params or SplatParams()
    n = sum(o.count for o in objects)
    eyes = len(camera.eyes)
    names = ("keys",) if pass_ == "keys" else tuple(outputs)
    if out is None:
        out = _alloc_outputs(names, n, eyes, device)
    objs, keep = _c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    c = ctx or default_context(0)
    c.call("rdx_project", objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), sort_bits,
           _abi.RDX_PASS_KEYS if pass_ == "keys" else _abi.RDX_PASS_FULL, 1 if cull_keys else 0,
           ctypes.byref(_c_outputs(out)))
    del keep
    return out


PROJECTION_METHODS = {"ewa": _abi.RDX_METHOD_EWA, "3dgut": _abi.RDX_METHOD_3DGUT, "htgs": _abi.RDX_METHOD_HTGS,
                      "raygs": _abi.RDX_METHOD_RAYGS}


def method_words(method, eyes):
    """Words per splat of a projection method ("ewa", "3dgut", "htgs",
    "raygs") with 1 or 2 eyes: ProjectionDef.headWords + eyes * eyeWords."""
    w = _abi.lib().rdx_method_words(PROJECTION_METHODS[method], eyes)
    if w < 0:
        raise ValueError(f"{method!r} with {eyes} eyes")
    return w


def project_words(objects, camera, method, params=None, sort_bits=24, cull_keys=True, ctx=None, out=None):
    """projectCollection with any projection method: {'words': uint32
    [n][method_words(method, E)] (head words, then each eye's), 'keys':
    uint32 [n]} as CUDA tensors (or into `out`). The ray methods take CUDA
    tables of the raw, ext or packed layout whose object-to-head transforms
    are a rotation times a uniform scale."""
    torch = _torch()
    n = sum(o.count for o in objects)
    if out is None:
        dev = torch.device("cuda", torch.cuda.current_device())
        out = {"words": torch.zeros((n, method_words(method, len(camera.eyes))), dtype=torch.int32, device=dev),
               "keys": torch.zeros(n, dtype=torch.int32, device=dev)}
    params = params or SplatParams()
    objs, keep = _c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    c = ctx or default_context(0)
    c.call("rdx_project_words", objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), PROJECTION_METHODS[method],
           sort_bits, 1 if cull_keys else 0, ctypes.c_void_p(_ptr(out.get("words"))), ctypes.c_void_p(_ptr(out.get("keys"))))
    del keep
    return out


def frame(objects, camera, params=None, sort_bits=24, outputs=DEFAULT_OUTPUTS, device="cuda", ctx=None,
          out=None, ordering=None, visible=None):
    """One frame: the projection (keys of splats culled in every eye invalid)
    and the stable back-to-front order. Returns the outputs plus 'ordering'
    ([n]: drawn splats first, culled ones after in index order) and 'visible'
    (an int; or, when `visible` is a 1-element device tensor, that tensor, and
    the call returns without waiting for the GPU)."""
    params = params or SplatParams()
    n = sum(o.count for o in objects)
    eyes = len(camera.eyes)
    if out is None:
        out = _alloc_outputs(tuple(outputs), n, eyes, device)
    if ordering is None:
        ordering = _alloc_outputs(("keys",), n, 1, device)["keys"]
    vis_host = ctypes.c_uint32(0) if visible is None else None
    objs, keep = _c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    c = ctx or default_context(0)
    c.call("rdx_frame", objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), sort_bits,
           ctypes.byref(_c_outputs(out)), _ptr(ordering),
           ctypes.byref(vis_host) if vis_host is not None else ctypes.c_void_p(_ptr(visible)))
    del keep
    res = dict(out)
    res["ordering"] = ordering
    res["visible"] = vis_host.value if vis_host is not None else visible
    return res


GRAD_OUTPUTS = ("mean2d", "conic", "depth", "opacity", "rgb")


def project_backward(objects, camera, upstream, fwd_opacity, params=None, ctx=None, grads=None):
    """The gradient of `project_collection`'s full pass (raw tables, CUDA
    tensors): upstream = {output: dL/d(output)} laid out as the forward's
    outputs (missing: zero), fwd_opacity = the forward's 'opacity' output.
    Returns one dict per object: centers [count][3], log_scales [count][3],
    quats [count][4], opacities [count], colors [count][1+K][3] (float32)."""
    torch = _torch()
    params = params or SplatParams()
    if grads is None:
        grads = []
        for o in objects:
            dev = torch.device("cuda", torch.cuda.current_device())
            k = (int(o.table.c.sh_degree) + 1) ** 2
            grads.append({"centers": torch.empty((o.count, 3), device=dev), "log_scales": torch.empty((o.count, 3), device=dev),
                          "quats": torch.empty((o.count, 4), device=dev), "opacities": torch.empty(o.count, device=dev),
                          "colors": torch.empty((o.count, k, 3), device=dev)})
    gin = _abi.rdx_grads_in()
    for name in GRAD_OUTPUTS:
        if upstream.get(name) is not None:
            setattr(gin, name, _ptr(upstream[name]))
    gin.fwd_opacity = _ptr(fwd_opacity)
    gout = (_abi.rdx_table_grads * max(1, len(objects)))()
    for i, g in enumerate(grads):
        for name, t in g.items():
            setattr(gout[i], name, _ptr(t))
    objs, keep = _c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    c = ctx or default_context(0)
    c.call("rdx_project_backward", objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), ctypes.byref(gin), gout)
    del keep
    return grads


def _c_views(views):
    """views: [(objects, camera)] -> (rdx_view array, objects kept alive)."""
    arr = (_abi.rdx_view * len(views))()
    keep = []
    for v, (objects, camera) in enumerate(views):
        objs, k = _c_objects(objects)
        cam = camera.to_c(_abi)
        keep += [objs, k, cam]
        arr[v].objects = ctypes.cast(objs, ctypes.POINTER(_abi.rdx_object))
        arr[v].n_objects = len(objects)
        arr[v].camera = ctypes.pointer(cam)
    return arr, keep


def _batch_rows(views):
    n = sum(o.count for objects, _ in views for o in objects)
    eyes = len(views[0][1].eyes)
    return n, eyes


def frame_batched(views, params=None, sort_bits=24, outputs=DEFAULT_OUTPUTS, device="cuda", ctx=None,
                  out=None, ordering=None, visible=None):
    """Several frames at once: views = [(objects, camera)]. View v's splats
    are rows first_v .. first_v + n_v - 1 of the outputs (eye e of row r at
    [e][r]); 'ordering'[first_v + i] is view v's i-th splat back to front (an
    index within the view) and 'visible'[v] its drawn count. Same results as
    one `frame` per view, in one projection launch per table kind and one
    segmented sort."""
    torch = _torch()
    params = params or SplatParams()
    n, eyes = _batch_rows(views)
    if out is None:
        out = _alloc_outputs(tuple(outputs), n, eyes, device)
    if ordering is None:
        ordering = _alloc_outputs(("keys",), n, 1, device)["keys"]
    if visible is None:
        visible = torch.zeros(len(views), dtype=torch.int32, device=device) if device is not None \
            else np.zeros(len(views), dtype=np.uint32)
    arr, keep = _c_views(views)
    prm = params.to_c()
    c = ctx or default_context(0)
    c.call("rdx_frame_batched", arr, len(views), ctypes.byref(prm), sort_bits, ctypes.byref(_c_outputs(out)),
           _ptr(ordering), _ptr(visible))
    del keep
    res = dict(out)
    res["ordering"] = ordering
    res["visible"] = visible
    return res


class Batch:
    """A batched frame captured once in a CUDA graph: `launch()` replays it
    (one cudaGraphLaunch); `update(views)` swaps cameras, object matrices and
    params for later launches. Everything lives in device memory."""

    def __init__(self, views, params=None, sort_bits=24, outputs=DEFAULT_OUTPUTS, device="cuda", ctx=None):
        torch = _torch()
        self.ctx = ctx or default_context(0)
        self.sort_bits = sort_bits
        n, eyes = _batch_rows(views)
        self.out = _alloc_outputs(tuple(outputs), n, eyes, device)
        self.ordering = torch.empty(n, dtype=torch.int32, device=device)
        self.visible = torch.zeros(len(views), dtype=torch.int32, device=device)
        self._views = views
        arr, keep = _c_views(views)
        prm = (params or SplatParams()).to_c()
        h = ctypes.c_void_p()
        self.ctx.call("rdx_batch_create", arr, len(views), ctypes.byref(prm), sort_bits, ctypes.byref(_c_outputs(self.out)),
                      _ptr(self.ordering), _ptr(self.visible), ctypes.byref(h))
        del keep
        self.handle = h

    def _call(self, name, *args):
        self.ctx._bind_stream()  # the batch runs on its context's stream
        _abi.check(getattr(_abi.lib(), name)(self.handle, *args), self.ctx.handle)

    def update(self, views, params=None):
        arr, keep = _c_views(views)
        prm = (params or SplatParams()).to_c()
        self._call("rdx_batch_update", arr, len(views), ctypes.byref(prm))
        del keep

    def launch(self):
        self._call("rdx_batch_launch")

    def synchronize(self):
        self._call("rdx_batch_synchronize")

    def launches(self):
        n = ctypes.c_uint64(0)
        self._call("rdx_batch_launches", ctypes.byref(n))
        return n.value

    def tune(self, reps=5):
        """Time projection block sizes and digit-pass variants on this batch,
        capture its graph again with the fastest and remember the choice in the
        context; returns the timings (the defaults are candidate 0)."""
        r = _abi.rdx_tune_result()
        self._call("rdx_batch_tune", int(reps), ctypes.byref(r))
        return r.as_dict()

    def results(self):
        res = dict(self.out)
        res["ordering"] = self.ordering
        res["visible"] = self.visible
        return res

    def close(self):
        if self.handle:
            _abi.lib().rdx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PLY_KINDS = ("standard", "points", "compressed")


def _bytes_arg(data):
    """(pointer, size, keep-alive) of file bytes: bytes / bytearray / numpy uint8 / a uint8 tensor."""
    if _is_torch(data):
        return _ptr(data), int(data.numel() * data.element_size()), data
    arr = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    return arr.ctypes.data, int(arr.nbytes), arr


SPZ_CONTAINERS = ("gzip", "ngsp")


def spz_info(data, ctx=None):
    """unpackSpz's view of an SPZ file's header (host bytes): {count, version,
    sh_degree, fractional_bits, flags, container}."""
    c = ctx or default_context(0)
    if _is_torch(data) and data.is_cuda:
        raise RadixError(_abi.RDX_ERR_ARG, "SPZ bytes must be in host memory (the container is unpacked on the host)")
    ptr, size, keep = _bytes_arg(data)
    info = _abi.rdx_spz_info()
    c.call("rdx_spz_read_info", ctypes.c_void_p(ptr), size, ctypes.byref(info))
    del keep
    return {"count": int(info.count), "version": int(info.version), "sh_degree": int(info.sh_degree),
            "fractional_bits": int(info.fractional_bits), "flags": int(info.flags),
            "container": SPZ_CONTAINERS[info.container]}


def decode_spz(data, sh_degree=-1, device="cuda", ctx=None):
    """SpzFile.read (src/core/spz.ts) of an SPZ file (host bytes, gzip or SPZ 4)
    decoded on the GPU into a raw Table of float32 columns (centres, ln scales,
    normalised quaternions, opacities, base rgb + SH of degree sh_degree, -1:
    the file's)."""
    torch = _torch()
    info = spz_info(data, ctx)
    deg = info["sh_degree"] if sh_degree < 0 else sh_degree
    n = info["count"]
    dev = torch.device(device)
    cols = {"centers": torch.empty((n, 3), device=dev), "log_scales": torch.empty((n, 3), device=dev),
            "quats": torch.empty((n, 4), device=dev), "opacities": torch.empty(n, device=dev),
            "colors": torch.empty((n, (deg + 1) ** 2, 3), device=dev)}
    c = ctx or default_context(0)
    ptr, size, keep = _bytes_arg(data)
    c.call("rdx_decode_spz", ctypes.c_void_p(ptr), size, deg, *(ctypes.c_void_p(_ptr(cols[k])) for k in
                                                                  ("centers", "log_scales", "quats", "opacities",
                                                                   "colors")))
    del keep
    return Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"], deg), cols


def rdxfile_info(data, ctx=None):
    """An RDX file's header (src/core/rdx.ts): {count, chunk_size, chunks,
    channels: [(bundle, label, format, element_bytes)] in payload order,
    header: the header's JSON as a dict}. Host bytes only."""
    import json
    c = ctx or default_context(0)
    if _is_torch(data) and data.is_cuda:
        raise RadixError(_abi.RDX_ERR_ARG, "RDX bytes must be in host memory (the payloads are inflated on the host)")
    ptr, size, keep = _bytes_arg(data)
    info = _abi.rdx_rdxfile_info()
    c.call("rdx_rdxfile_read_info", ctypes.c_void_p(ptr), size, ctypes.byref(info), None, 0, None, 0)
    chans = (_abi.rdx_rdxfile_channel * max(info.n_channels, 1))()
    text = ctypes.create_string_buffer(int(info.header_json_bytes) + 1)
    c.call("rdx_rdxfile_read_info", ctypes.c_void_p(ptr), size, ctypes.byref(info), chans, info.n_channels, text,
           info.header_json_bytes)
    del keep
    channels = [(ch.bundle.decode(), ch.label.decode(), ch.format.decode(), int(ch.element_bytes))
                for ch in chans[:info.n_channels]]
    return {"count": int(info.count), "chunk_size": int(info.chunk_size), "chunks": int(info.n_chunks),
            "channels": channels, "header": json.loads(text.raw[:info.header_json_bytes].decode())}


def decode_rdxfile(data, device="cuda", ctx=None):
    """RdxFile.read of a whole RDX file (host bytes): (info, {bundle: {label:
    uint8 tensor [count, element_bytes]}}), every serialized channel decoded
    on the GPU (inflated on the host, bytes transposed back on the device)."""
    torch = _torch()
    info = rdxfile_info(data, ctx)
    n = info["count"]
    dev = torch.device(device)
    out, ptrs = {}, []
    for bundle, label, fmt, eb in info["channels"]:
        t = torch.empty((n, eb), dtype=torch.uint8, device=dev)
        out.setdefault(bundle, {})[label] = t
        ptrs.append(_ptr(t) if n else None)
    c = ctx or default_context(0)
    ptr, size, keep = _bytes_arg(data)
    arr = (ctypes.c_void_p * max(len(ptrs), 1))(*ptrs)
    c.call("rdx_decode_rdxfile", ctypes.c_void_p(ptr), size, arr)
    del keep
    return info, out


def _words(t):
    """A uint8 [count, 16] channel as int32 [count, 4] words."""
    return t.view(_torch().int32).reshape(t.shape[0], -1)


def rdxfile_table(data, device="cuda", ctx=None, palette=None):
    """A Table over an RDX file's splats: its extSplats, covSplats or
    packedSplats bundle (src/core/splats.ts:69-77; packedSplats' meta.encoding)
    and its SH: a per-splat bundle ("extSh" or "packedSh", meta {codec,
    degree}, src/core/sh.ts:230-240), or labels (bundle shLabel) into the
    ShPalette that `palette` (the palette's own RDX file) holds (bundle
    shPalette, meta {codec, degree, size, stride}, src/core/sh.ts:426-470).
    Decoded on the GPU. Returns (table, channels)."""
    info, ch = decode_rdxfile(data, device, ctx)
    bundles = info["header"]["bundles"]
    sh, deg, codec, pal = (), 0, "ext", None
    for name in ("extSh", "packedSh"):
        if name in ch:
            meta = bundles[name].get("meta", {})
            codec = meta.get("codec", name[:-2])
            deg = int(meta.get("degree", 0))
            sh = [_words(t) for t in ch[name].values()]
            break
    if palette is not None:
        if "shLabel" not in ch:
            raise RadixError(_abi.RDX_ERR_ARG, "a palette was given but the RDX file has no shLabel bundle")
        pinfo, pch = decode_rdxfile(palette, device, ctx)
        if "shPalette" not in pch or "shEntries" not in pch["shPalette"]:
            raise RadixError(_abi.RDX_ERR_ARG, "Not an SH palette: no shPalette.shEntries channel")
        meta = pinfo["header"]["bundles"]["shPalette"].get("meta", {})
        codec, deg = meta.get("codec", "ext"), int(meta.get("degree", 0))
        labels = ch["shLabel"]["label"].view(_torch().int16).reshape(-1)
        pal = (_words(pch["shPalette"]["shEntries"]), labels, int(meta["stride"]))
        ch["shPalette"] = pch["shPalette"]
    kw = {"palette": pal} if pal is not None else {}
    if "extSplats" in ch:
        t = Table.ext(_words(ch["extSplats"]["extA"]), _words(ch["extSplats"]["extB"]), sh, deg, codec, **kw)
    elif "covSplats" in ch:
        t = Table.cov(_words(ch["covSplats"]["covA"]), _words(ch["covSplats"]["covB"]), sh, deg, codec, **kw)
    elif "packedSplats" in ch:
        e = dict(zip(("rgbMin", "rgbMax", "lnScaleMin", "lnScaleMax"), Table.PACKED_ENCODING))
        e.update(bundles["packedSplats"].get("meta", {}).get("encoding", {}))
        enc = (e["rgbMin"], e["rgbMax"], e["lnScaleMin"], e["lnScaleMax"])
        t = Table.packed(_words(ch["packedSplats"]["packed"]), enc, sh, deg, codec, **kw)
    else:
        raise RadixError(_abi.RDX_ERR_ARG, "the RDX file has no extSplats, covSplats or packedSplats bundle")
    return t, ch


def ply_info(data, ctx=None):
    """PlyFile.read's view of a file's header: {count, sh_degree, kind}."""
    c = ctx or default_context(0)
    ptr, size, keep = _bytes_arg(data)
    info = _abi.rdx_ply_info()
    c.call("rdx_ply_read_info", ctypes.c_void_p(ptr), size, ctypes.byref(info))
    del keep
    return {"count": int(info.count), "sh_degree": int(info.sh_degree), "kind": PLY_KINDS[info.kind]}


def decode_ply(data, sh_degree=-1, device="cuda", ctx=None):
    """PlyFile.read (src/core/ply.ts) of a binary PLY file (bytes or a CUDA
    uint8 tensor) decoded on the GPU into a raw Table of float32 columns
    (centres, ln scales, normalised quaternions, opacities, base rgb + SH of
    degree sh_degree, -1: the file's)."""
    torch = _torch()
    info = ply_info(data, ctx)
    deg = info["sh_degree"] if sh_degree < 0 else sh_degree
    n = info["count"]
    dev = torch.device(device)
    cols = {"centers": torch.empty((n, 3), device=dev), "log_scales": torch.empty((n, 3), device=dev),
            "quats": torch.empty((n, 4), device=dev), "opacities": torch.empty(n, device=dev),
            "colors": torch.empty((n, (deg + 1) ** 2, 3), device=dev)}
    c = ctx or default_context(0)
    ptr, size, keep = _bytes_arg(data)
    c.call("rdx_decode_ply", ctypes.c_void_p(ptr), size, deg, *(ctypes.c_void_p(_ptr(cols[k])) for k in
                                                                  ("centers", "log_scales", "quats", "opacities",
                                                                   "colors")))
    del keep
    return Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"], deg), cols
