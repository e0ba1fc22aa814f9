"""ctypes binding of the C ABI in include/aniso_b200.h (libaniso_b200.so, built in-tree).

The library is loaded on first use (the first call through `lib`, or `load()`), so that importing
the package -- for its pure-numpy scene generator, say -- maps no GPU code. There is no fallback:
if the library is missing, that first use raises ImportError with the command that builds it.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libaniso_b200.so")

OK = 0
ERR_ARGUMENT = 1
ERR_CUDA = 2
ERR_NO_DEVICE = 3
ERR_OUT_OF_MEMORY = 4
ERR_DEVICE_WAIT = 5
NOALLOC_MAX_GAUSSIANS = 65536   # ANISO_B200_NOALLOC_MAX_GAUSSIANS
NOALLOC_MAX_PAIRS = 1048576     # ANISO_B200_NOALLOC_MAX_PAIRS

# Every symbol include/aniso_b200.h declares.
EXPORTS = [
    "aniso_b200_available",
    "aniso_b200_scene_create",
    "aniso_b200_scene_create_raw",
    "aniso_b200_scene_destroy",
    "aniso_b200_render",
    "aniso_b200_render_device",
    "aniso_b200_sync",
    "aniso_b200_last_error",
    "aniso_b200_debug_projection",
    "aniso_b200_debug_sorted",
    "aniso_b200_sort_projection",
    "aniso_b200_profile",
    "aniso_b200_profile_read",
    "aniso_b200_frame_kernels",
    "aniso_b200_trainer_create",
    "aniso_b200_trainer_destroy",
    "aniso_b200_train_forward",
    "aniso_b200_train_backward",
    "aniso_b200_batch_create",
    "aniso_b200_batch_render",
    "aniso_b200_batch_sync",
    "aniso_b200_batch_destroy",
    "aniso_b200_train_batch_forward",
    "aniso_b200_train_batch_backward",
    "aniso_b200_sort_projection_noalloc",
    "aniso_b200_scene_load_ply",
    "aniso_b200_adam_step",
    "aniso_b200_colmap_load",
]


class Camera(ctypes.Structure):
    _fields_ = [("R", ctypes.c_double * 9), ("t", ctypes.c_double * 3), ("fx", ctypes.c_double),
                ("fy", ctypes.c_double), ("cx", ctypes.c_double), ("cy", ctypes.c_double),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32)]


class ColmapCamera(ctypes.Structure):
    _fields_ = [("camera", Camera), ("image_name", ctypes.c_char * 256)]


class Options(ctypes.Structure):
    _fields_ = [("sh_degree", ctypes.c_int32), ("splat_scale", ctypes.c_float)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("sh_degree", ctypes.c_int32), ("splat_scale", ctypes.c_float), ("tile_w", ctypes.c_int32),
                ("tile_h", ctypes.c_int32), ("blend_batch", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("radix_bits", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("visible", ctypes.c_uint64), ("tile_pairs", ctypes.c_uint64), ("project_ms", ctypes.c_double),
                ("sort_ms", ctypes.c_double), ("blend_ms", ctypes.c_double)]


class RawParams(ctypes.Structure):
    _fields_ = [("means", ctypes.c_void_p), ("log_scales", ctypes.c_void_p), ("quats", ctypes.c_void_p),
                ("opacity_logits", ctypes.c_void_p), ("sh", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("sh_degree", ctypes.c_int32)]


class RawGrads(ctypes.Structure):
    _fields_ = [("means", ctypes.c_void_p), ("log_scales", ctypes.c_void_p), ("quats", ctypes.c_void_p),
                ("opacity_logits", ctypes.c_void_p), ("sh", ctypes.c_void_p), ("grad2d", ctypes.c_void_p),
                ("visible", ctypes.c_void_p), ("fresh", ctypes.c_int32)]


class AdamGroup(ctypes.Structure):
    _fields_ = [("param", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("exp_avg", ctypes.c_void_p),
                ("exp_avg_sq", ctypes.c_void_p), ("count", ctypes.c_int64), ("lr", ctypes.c_float),
                ("lr_head", ctypes.c_float), ("row", ctypes.c_int32), ("head", ctypes.c_int32), ("eps", ctypes.c_float)]


class AnisoError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("aniso_b200 error %d: %s" % (code, message))
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("%s is missing: build it with `python aniso_b200/build.py`" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    I64, I32, U64 = ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64
    sig = {
        "aniso_b200_available": [ctypes.POINTER(I32)],
        "aniso_b200_scene_create": [P, P, I64, I32, ctypes.POINTER(P)],
        "aniso_b200_scene_create_raw": [P, P, P, P, P, P, I64, I32, ctypes.POINTER(P)],
        "aniso_b200_scene_destroy": [P],
        "aniso_b200_scene_load_ply": [ctypes.c_char_p, ctypes.POINTER(P)],
        "aniso_b200_adam_step": [ctypes.POINTER(AdamGroup), I32, I32, ctypes.c_float, ctypes.c_float, P],
        "aniso_b200_render": [P, ctypes.POINTER(Camera), ctypes.POINTER(Options), P, ctypes.POINTER(Stats)],
        "aniso_b200_render_device": [P, ctypes.POINTER(Camera), ctypes.POINTER(Options), P, P],
        "aniso_b200_sync": [P, ctypes.POINTER(Stats)],
        "aniso_b200_debug_projection": [P, ctypes.POINTER(Camera), ctypes.POINTER(Options), P, P, P, P, P, P],
        "aniso_b200_debug_sorted": [P, ctypes.POINTER(Camera), ctypes.POINTER(Options), P, P, U64, P,
                                    ctypes.POINTER(U64)],
        "aniso_b200_sort_projection": [I64, P, P, P, I32, I32, P, P, U64, P, ctypes.POINTER(U64)],
        "aniso_b200_profile": [P, I32],
        "aniso_b200_trainer_create": [ctypes.POINTER(P)],
        "aniso_b200_trainer_destroy": [P],
        "aniso_b200_train_forward": [P, ctypes.POINTER(RawParams), ctypes.POINTER(Camera), ctypes.POINTER(Options), P,
                                     P],
        "aniso_b200_train_backward": [P, P, ctypes.POINTER(RawGrads), P],
        "aniso_b200_batch_create": [P, I32, P, I32, ctypes.POINTER(BatchOptions), ctypes.POINTER(P)],
        "aniso_b200_batch_render": [P, P, P, P],
        "aniso_b200_batch_sync": [P, ctypes.POINTER(Stats)],
        "aniso_b200_batch_destroy": [P],
        "aniso_b200_train_batch_forward": [P, P, I32, P, P, I32, ctypes.POINTER(BatchOptions), P, P],
        "aniso_b200_train_batch_backward": [P, P, P, P],
        "aniso_b200_sort_projection_noalloc": [I64, P, P, P, I32, I32, P, P, U64, P, P, P],
        "aniso_b200_profile_read": [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(I64)],
        "aniso_b200_frame_kernels": [P, ctypes.POINTER(ctypes.c_int32)],
        "aniso_b200_colmap_load": [ctypes.c_char_p, ctypes.POINTER(ColmapCamera), I32, ctypes.POINTER(I32)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.aniso_b200_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.aniso_b200_last_error.restype = ctypes.c_size_t
    return lib


class _LazyLibrary:
    """Stands in for the ctypes library until its first attribute lookup, which loads it."""

    def __init__(self):
        self._lib = None

    def load(self):
        if self._lib is None:
            self._lib = _load()
        return self._lib

    def __getattr__(self, name):
        return getattr(self.load(), name)


lib = _LazyLibrary()


def load():
    """Loads libaniso_b200.so now (raises ImportError if it is missing) and returns it."""
    return lib.load()


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.aniso_b200_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != OK:
        raise AnisoError(rc, last_error())
