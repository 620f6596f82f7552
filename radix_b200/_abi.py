"""ctypes binding of include/radix_b200.h.

The structures mirror the C header field for field. The library is the
in-tree build radix_b200/lib/libradix_b200.so; loading fails loudly when it is
missing (there is no CPU fallback for any entry point).
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# RADIX_B200_CHECK=1 loads the bounds-checked build (radix_b200/build.py --check)
LIB_PATH = os.path.join(HERE, "lib", "libradix_b200_check.so" if os.environ.get("RADIX_B200_CHECK") == "1"
                        else "libradix_b200.so")

RDX_OK = 0
RDX_ERR_ARG = 1
RDX_ERR_CAPACITY = 2
RDX_ERR_CUDA = 3
RDX_ERR_TIMEOUT = 4
RDX_ERR_UNSUPPORTED = 5
RDX_ERR_NOMEM = 6

RDX_LAYOUT_RAW = 0
RDX_LAYOUT_EXT = 1
RDX_LAYOUT_PACKED = 2
RDX_LAYOUT_COV = 3
RDX_SH_EXT = 0
RDX_SH_PACKED = 1
RDX_DTYPE_F32 = 0
RDX_DTYPE_F16 = 1
RDX_PASS_FULL = 0
RDX_PASS_KEYS = 1
RDX_METHOD_EWA = 0
RDX_METHOD_3DGUT = 1
RDX_METHOD_HTGS = 2
RDX_METHOD_RAYGS = 3
RDX_PHASE_PROJECT = 0
RDX_PHASE_SORT = 1
RDX_PHASE_COPY_IN = 2
RDX_PHASE_COPY_OUT = 3
RDX_PHASE_BATCH = 4
RDX_PHASES = 5

c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)


class rdx_table(ctypes.Structure):
    _fields_ = [
        ("layout", ctypes.c_int32),
        ("sh_degree", ctypes.c_int32),
        ("color_dtype", ctypes.c_int32),
        ("sh_codec", ctypes.c_int32),
        ("count", ctypes.c_uint64),
        ("centers", ctypes.c_void_p),
        ("log_scales", ctypes.c_void_p),
        ("quats", ctypes.c_void_p),
        ("opacities", ctypes.c_void_p),
        ("colors", ctypes.c_void_p),
        ("ext_a", ctypes.c_void_p),
        ("ext_b", ctypes.c_void_p),
        ("ext_sh", ctypes.c_void_p * 6),
        ("packed", ctypes.c_void_p),
        ("packed_encoding", ctypes.c_float * 4),
        ("sh_palette", ctypes.c_void_p),
        ("sh_label", ctypes.c_void_p),
        ("sh_stride", ctypes.c_uint32),
        ("sh_palette_size", ctypes.c_uint32),
    ]


class rdx_params(ctypes.Structure):
    _fields_ = [
        ("max_std_dev", ctypes.c_float),
        ("min_alpha", ctypes.c_float),
        ("falloff", ctypes.c_float),
        ("lod_inflate", ctypes.c_int32),
        ("blur_amount", ctypes.c_float),
        ("pre_blur_amount", ctypes.c_float),
        ("clip_xy", ctypes.c_float),
        ("min_pixel_radius", ctypes.c_float),
        ("max_pixel_radius", ctypes.c_float),
        ("min_contribution", ctypes.c_float),
        ("focal_distance", ctypes.c_float),
        ("aperture_tan", ctypes.c_float),
        ("sort_guard", ctypes.c_float),
        ("max_sh_degree", ctypes.c_int32),
    ]


class rdx_eye(ctypes.Structure):
    _fields_ = [
        ("view", ctypes.c_double * 16),
        ("projection", ctypes.c_double * 16),
        ("ortho", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class rdx_camera(ctypes.Structure):
    _fields_ = [
        ("head", ctypes.c_double * 16),
        ("eyes", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("eye", rdx_eye * 2),
        ("width", ctypes.c_double),
        ("height", ctypes.c_double),
        ("ndc_z_min", ctypes.c_double),
    ]


class rdx_object(ctypes.Structure):
    _fields_ = [
        ("table", ctypes.POINTER(rdx_table)),
        ("count", ctypes.c_uint64),
        ("world", ctypes.c_double * 16),
        ("params", ctypes.POINTER(rdx_params)),
    ]


class rdx_view(ctypes.Structure):
    _fields_ = [
        ("objects", ctypes.POINTER(rdx_object)),
        ("n_objects", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("camera", ctypes.POINTER(rdx_camera)),
    ]


class rdx_grads_in(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("mean2d", "conic", "depth", "opacity", "rgb", "fwd_opacity")]


class rdx_table_grads(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("centers", "log_scales", "quats", "opacities", "colors")]


class rdx_ply_info(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("sh_degree", ctypes.c_int32), ("kind", ctypes.c_int32)]


class rdx_spz_info(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("version", ctypes.c_int32), ("sh_degree", ctypes.c_int32),
                ("fractional_bits", ctypes.c_int32), ("flags", ctypes.c_int32), ("container", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class rdx_rdxfile_info(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("chunk_size", ctypes.c_uint64), ("n_chunks", ctypes.c_int32),
                ("n_channels", ctypes.c_int32), ("header_json_bytes", ctypes.c_uint64)]


class rdx_rdxfile_channel(ctypes.Structure):
    _fields_ = [("bundle", ctypes.c_char * 64), ("label", ctypes.c_char * 64), ("format", ctypes.c_char * 16),
                ("element_bytes", ctypes.c_int32), ("reserved", ctypes.c_int32)]


RDX_TUNE_MAX = 16


class rdx_tune_result(ctypes.Structure):
    _fields_ = [
        ("sort_variant", ctypes.c_int32),
        ("project_warps", ctypes.c_int32),
        ("candidates", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("default_ms", ctypes.c_double),
        ("tuned_ms", ctypes.c_double),
        ("cand_sort", ctypes.c_int32 * RDX_TUNE_MAX),
        ("cand_warps", ctypes.c_int32 * RDX_TUNE_MAX),
        ("cand_ms", ctypes.c_double * RDX_TUNE_MAX),
    ]

    def as_dict(self):
        return {"sort_variant": self.sort_variant, "project_warps": self.project_warps,
                "default_ms": self.default_ms, "tuned_ms": self.tuned_ms,
                "candidates": [{"sort_variant": self.cand_sort[i], "project_warps": self.cand_warps[i],
                                "ms": self.cand_ms[i]} for i in range(self.candidates)]}


class rdx_outputs(ctypes.Structure):
    _fields_ = [
        ("mean2d", ctypes.c_void_p),
        ("conic", ctypes.c_void_p),
        ("depth", ctypes.c_void_p),
        ("opacity", ctypes.c_void_p),
        ("rgb", ctypes.c_void_p),
        ("radii", ctypes.c_void_p),
        ("words", ctypes.c_void_p),
        ("keys", ctypes.c_void_p),
    ]


# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "rdx_version": (ctypes.c_int, []),
    "rdx_params_default": (None, [ctypes.POINTER(rdx_params)]),
    "rdx_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "rdx_ctx_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rdx_ctx_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_ctx_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "rdx_ctx_reserve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "rdx_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "rdx_ctx_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rdx_ctx_set_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int]),
    "rdx_ctx_set_sort_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rdx_batch_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "rdx_sort_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p]),
    "rdx_ctx_phase_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_ctx_launches": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_ctx_set_host_reads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rdx_ctx_host_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_sort_keys_compute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]),
    "rdx_sort_keys_compute_f32": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]),
    "rdx_sort": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_uint64, ctypes.c_void_p]),
    "rdx_sort_pairs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]),
    "rdx_sort_pairs_indirect": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_uint64, ctypes.c_int]),
    "rdx_compact": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_splat_sort": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_project": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_object), ctypes.c_int, ctypes.POINTER(rdx_camera),
                                   ctypes.POINTER(rdx_params), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(rdx_outputs)]),
    "rdx_sort_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_frame": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_object), ctypes.c_int, ctypes.POINTER(rdx_camera),
                                 ctypes.POINTER(rdx_params), ctypes.c_int, ctypes.POINTER(rdx_outputs), ctypes.c_void_p,
                                 ctypes.c_void_p]),
    "rdx_method_words": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "rdx_project_words": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_object), ctypes.c_int,
                                         ctypes.POINTER(rdx_camera), ctypes.POINTER(rdx_params), ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_project_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_object), ctypes.c_int,
                                            ctypes.POINTER(rdx_camera), ctypes.POINTER(rdx_params),
                                            ctypes.POINTER(rdx_grads_in), ctypes.POINTER(rdx_table_grads)]),
    "rdx_ply_read_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(rdx_ply_info)]),
    "rdx_decode_ply": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_spz_read_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(rdx_spz_info)]),
    "rdx_decode_spz": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_rdxfile_read_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                             ctypes.POINTER(rdx_rdxfile_info), ctypes.POINTER(rdx_rdxfile_channel),
                                             ctypes.c_int, ctypes.c_char_p, ctypes.c_uint64]),
    "rdx_decode_rdxfile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "rdx_frame_batched": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_view), ctypes.c_int, ctypes.POINTER(rdx_params),
                                         ctypes.c_int, ctypes.POINTER(rdx_outputs), ctypes.c_void_p, ctypes.c_void_p]),
    "rdx_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_view), ctypes.c_int, ctypes.POINTER(rdx_params),
                                        ctypes.c_int, ctypes.POINTER(rdx_outputs), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "rdx_batch_update": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(rdx_view), ctypes.c_int, ctypes.POINTER(rdx_params)]),
    "rdx_batch_launch": (ctypes.c_int, [ctypes.c_void_p]),
    "rdx_batch_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "rdx_batch_launches": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "rdx_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
}

_lib = None


def lib():
    """The loaded C library (raises when the build is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"radix_b200: the CUDA library {LIB_PATH} is not built; run __graft_entry__.build() "
                "(there is no CPU fallback)")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class RadixError(RuntimeError):
    """A failed C-ABI call: .code is the RDX_* status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


def check(status, ctx_handle=None):
    if status != RDX_OK:
        msg = lib().rdx_last_error(ctx_handle).decode() if ctx_handle else ""
        raise RadixError(status, msg or f"radix_b200 status {status}")
