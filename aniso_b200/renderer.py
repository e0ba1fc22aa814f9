"""Python mirror of the reference's GPU renderer interface, aniso::GpuRenderer
(include/aniso/gpu_render.h:22-37), over the C ABI of libaniso_b200.so.

    r = GpuRenderer(gaussians, sh, sh_degree)     # GpuRenderer(const Scene&): uploads once
    img = r.render(camera, stats, options)        # Image render(const Camera&, RenderStats*, ...)
    GpuRenderer.available()                       # static bool available()

Errors raise AnisoError (the reference throws std::runtime_error, gpu_render.cu:18-21).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import struct

import numpy as np

from . import _lib
from ._lib import check, lib


@dataclasses.dataclass
class RenderOptions:
    """aniso::RenderOptions (render.h:28-33)."""

    sh_degree: int = 3
    splat_scale: float = 1.0

    def c(self) -> _lib.Options:
        return _lib.Options(int(self.sh_degree), float(self.splat_scale))


# The default options, packed once (the library only reads them).
_DEFAULT_OPTIONS = RenderOptions().c()

_CAM_LAYOUT = struct.Struct("16d2i")  # R (row-major), t, fx, fy, cx, cy as double; width, height
assert _CAM_LAYOUT.size == ctypes.sizeof(_lib.Camera)


def c_camera(cam) -> _lib.Camera:
    """aniso_b200_camera of a camera (R, t, fx, fy, cx, cy, width, height), packed in one copy."""
    r = np.asarray(cam.R, np.float64).reshape(9).tolist()
    t = np.asarray(cam.t, np.float64).reshape(3).tolist()
    return _lib.Camera.from_buffer_copy(_CAM_LAYOUT.pack(*r, *t, cam.fx, cam.fy, cam.cx, cam.cy, cam.width,
                                                          cam.height))


def _ply_shape(path):
    """(Gaussians, SH degree) from a PLY header (the library has already validated it)."""
    n, rest = 0, 0
    with open(path, "rb") as f:
        for raw in f:
            line = raw.decode("ascii", "replace").strip()
            if line.startswith("element vertex"):
                n = int(line.split()[2])
            elif line.startswith("property") and line.split()[-1].startswith("f_rest_"):
                rest += 1
            elif line == "end_header":
                break
    deg = {0: 0, 9: 1, 24: 2, 45: 3, 72: 4}[rest]
    return n, deg


def _ptr(a: np.ndarray) -> int:
    """Address of a C-contiguous array's data, for a c_void_p argument (the caller keeps `a` alive)."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _stats_dict(s: _lib.Stats) -> dict:
    return {"visible": int(s.visible), "tile_pairs": int(s.tile_pairs), "project_ms": s.project_ms,
            "sort_ms": s.sort_ms, "blend_ms": s.blend_ms}


class GpuRenderer:
    def __init__(self, gaussians: np.ndarray, sh: np.ndarray, sh_degree: int):
        g = np.ascontiguousarray(gaussians, np.float32)
        s = np.ascontiguousarray(sh, np.float32)
        n = g.shape[0]
        if g.shape != (n, 11):
            raise ValueError("gaussians must be (n, 11)")
        if s.size != n * (sh_degree + 1) ** 2 * 3:
            raise ValueError("sh must hold n * (degree+1)^2 * 3 floats")
        self._h = ctypes.c_void_p()
        check(lib.aniso_b200_scene_create(_ptr(g), _ptr(s), n, sh_degree, ctypes.byref(self._h)))
        self.n = n
        self.sh_degree = sh_degree

    @classmethod
    def from_raw(cls, raw) -> "GpuRenderer":
        """Uploads a scene in the PLY's raw form and activates it on the device."""
        self = cls.__new__(cls)
        f = lambda a: np.ascontiguousarray(a, np.float32)
        xyz, dc, rest, op, sc, rot = f(raw.xyz), f(raw.f_dc), f(raw.f_rest), f(raw.opacity), f(raw.scale), f(raw.rot)
        self._h = ctypes.c_void_p()
        check(lib.aniso_b200_scene_create_raw(_ptr(xyz), _ptr(dc), _ptr(rest), _ptr(op), _ptr(sc), _ptr(rot), raw.n,
                                              raw.sh_degree, ctypes.byref(self._h)))
        self.n = raw.n
        self.sh_degree = raw.sh_degree
        return self

    @classmethod
    def from_ply(cls, path) -> "GpuRenderer":
        """Loads a 3DGS PLY like aniso::loadPly, with the de-interleave and activation on the device."""
        self = cls.__new__(cls)
        self._h = ctypes.c_void_p()
        check(lib.aniso_b200_scene_load_ply(os.fsencode(path), ctypes.byref(self._h)))
        n, deg = _ply_shape(path)
        self.n = n
        self.sh_degree = deg
        return self

    @staticmethod
    def available() -> bool:
        a = ctypes.c_int32(0)
        check(lib.aniso_b200_available(ctypes.byref(a)))
        return bool(a.value)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.aniso_b200_scene_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, camera, stats: dict | None = None, options: RenderOptions | None = None,
               out: np.ndarray | None = None) -> np.ndarray:
        """RGB8 image (H, W, 3) in host memory; fills `stats` like RenderStats if given."""
        o = options.c() if options is not None else _DEFAULT_OPTIONS
        c = c_camera(camera)
        if out is None:
            out = np.empty((camera.height, camera.width, 3), np.uint8)
        assert out.shape == (camera.height, camera.width, 3) and out.dtype == np.uint8
        st = _lib.Stats() if stats is not None else None
        check(lib.aniso_b200_render(self._h, ctypes.byref(c), ctypes.byref(o), _ptr(out),
                                    ctypes.byref(st) if st is not None else None))
        if stats is not None:
            stats.update(_stats_dict(st))
        return out

    def render_device(self, camera, rgb_device_ptr: int, stream_ptr: int = 0,
                      options: RenderOptions | None = None):
        """Enqueues a render into device memory on a CUDA stream; no wait."""
        o = (options or RenderOptions()).c()
        c = c_camera(camera)
        check(lib.aniso_b200_render_device(self._h, ctypes.byref(c), ctypes.byref(o), ctypes.c_void_p(rgb_device_ptr),
                                           ctypes.c_void_p(stream_ptr)))

    def profile(self, enable: bool = True):
        """Starts (clearing the totals) or stops per-stage event timing of render_device frames."""
        check(lib.aniso_b200_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        """Summed stage times (ms) of the profiled render_device frames, and their count."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        f = ctypes.c_int64()
        check(lib.aniso_b200_profile_read(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(f)))
        return {"project_ms": a.value, "sort_ms": b.value, "blend_ms": c.value, "frames": f.value}

    def frame_kernels(self) -> int:
        """Kernels the last render / render_device frame launched (the library's own)."""
        k = ctypes.c_int32()
        check(lib.aniso_b200_frame_kernels(self._h, ctypes.byref(k)))
        return k.value

    def sync(self) -> dict:
        st = _lib.Stats()
        check(lib.aniso_b200_sync(self._h, ctypes.byref(st)))
        return _stats_dict(st)

    def debug_projection(self, camera, options: RenderOptions | None = None) -> dict:
        """Per-Gaussian projection in the reference kernel's layout (gpu_render.cu:86-88)."""
        n = self.n
        o = (options or RenderOptions()).c()
        c = c_camera(camera)
        out = {"uv": np.zeros((n, 2), np.float32), "conic_opacity": np.zeros((n, 4), np.float32),
               "depth": np.zeros(n, np.float32), "rgb": np.zeros((n, 3), np.float32),
               "rect": np.zeros((n, 4), np.uint32), "tiles_touched": np.zeros(n, np.uint32)}
        check(lib.aniso_b200_debug_projection(self._h, ctypes.byref(c), ctypes.byref(o), _ptr(out["uv"]),
                                              _ptr(out["conic_opacity"]), _ptr(out["depth"]), _ptr(out["rgb"]),
                                              _ptr(out["rect"]), _ptr(out["tiles_touched"])))
        return out

    def debug_sorted(self, camera, options: RenderOptions | None = None, capacity: int | None = None):
        """(tile ids u32[P], Gaussian indices u32[P], ranges u32[T, 2]) after the sort."""
        o = (options or RenderOptions()).c()
        c = c_camera(camera)
        tiles_x = (camera.width + 15) // 16
        tiles_y = (camera.height + 15) // 16
        cap = capacity if capacity is not None else max(1, 64 * self.n + 1024)
        tiles = np.zeros(cap, np.uint32)
        values = np.zeros(cap, np.uint32)
        ranges = np.zeros((tiles_x * tiles_y, 2), np.uint32)
        pairs = ctypes.c_uint64(0)
        check(lib.aniso_b200_debug_sorted(self._h, ctypes.byref(c), ctypes.byref(o), _ptr(tiles), _ptr(values), cap,
                                          _ptr(ranges), ctypes.byref(pairs)))
        p = pairs.value
        return tiles[:p].copy(), values[:p].copy(), ranges


def sort_projection(tiles_touched, rect, depth, tiles_x: int, tiles_y: int):
    """The product's sort alone, on a projection given in the reference kernel's layout."""
    tt = np.ascontiguousarray(tiles_touched, np.uint32)
    rc = np.ascontiguousarray(rect, np.uint32).reshape(-1, 4)
    dp = np.ascontiguousarray(depth, np.float32)
    n = tt.shape[0]
    cap = max(1, int(tt.astype(np.int64).sum()))
    tiles = np.zeros(cap, np.uint32)
    values = np.zeros(cap, np.uint32)
    ranges = np.zeros((tiles_x * tiles_y, 2), np.uint32)
    pairs = ctypes.c_uint64(0)
    check(lib.aniso_b200_sort_projection(n, _ptr(tt), _ptr(rc), _ptr(dp), tiles_x, tiles_y, _ptr(tiles),
                                         _ptr(values), cap, _ptr(ranges), ctypes.byref(pairs)))
    p = pairs.value
    return tiles[:p].copy(), values[:p].copy(), ranges


def keys_of(tiles: np.ndarray, values: np.ndarray, depth: np.ndarray) -> np.ndarray:
    """The reference's 64-bit sort keys (tile << 32 | depth bits, gpu_render.cu:157) of a pair list."""
    bits = np.ascontiguousarray(depth, np.float32).view(np.uint32)
    return (tiles.astype(np.uint64) << np.uint64(32)) | bits[values].astype(np.uint64)


def colmap_load(folder) -> list:
    """aniso::loadColmapCameras through the C ABI (aniso_b200_colmap_load): the binary model when
    cameras.bin exists, else the text one; scenes.Camera objects sorted by image name."""
    from .scenes import Camera

    path = os.fsencode(folder)
    count = ctypes.c_int32(0)
    check(lib.aniso_b200_colmap_load(path, None, 0, ctypes.byref(count)))
    arr = (_lib.ColmapCamera * max(count.value, 1))()
    check(lib.aniso_b200_colmap_load(path, arr, count.value, ctypes.byref(count)))
    out = []
    for k in range(count.value):
        c = arr[k].camera
        out.append(Camera(c.width, c.height, c.fx, c.fy, c.cx, c.cy, np.array(c.R[:], np.float64).reshape(3, 3),
                          np.array(c.t[:], np.float64), arr[k].image_name.decode()))
    return out


@dataclasses.dataclass
class BatchOptions:
    """aniso_b200_batch_options: colour options plus the launch shape (tile, blend batch, graph,
    radix digit width)."""

    sh_degree: int = 3
    splat_scale: float = 1.0
    tile: tuple[int, int] = (16, 16)
    blend_batch: int = 256
    use_graph: bool = False
    radix_bits: int = 8

    def c(self) -> _lib.BatchOptions:
        return _lib.BatchOptions(int(self.sh_degree), float(self.splat_scale), int(self.tile[0]), int(self.tile[1]),
                                 int(self.blend_batch), 1 if self.use_graph else 0, int(self.radix_bits))


def c_cameras(cameras) -> ctypes.Array:
    arr = (_lib.Camera * len(cameras))()
    for k, cam in enumerate(cameras):
        arr[k] = c_camera(cam)
    return arr


class BatchRenderer:
    """Many views of several uploaded scenes in one launch sequence (aniso_b200_batch_*).

    view_scene[k] names the scene (an index into `scenes`) of view k; the views of one scene are
    consecutive. The scenes must stay alive as long as the batch.
    """

    def __init__(self, scenes: list[GpuRenderer], view_scene, options: BatchOptions | None = None):
        self.scenes = list(scenes)
        self.view_scene = np.ascontiguousarray(view_scene, np.int32)
        self.options = options or BatchOptions()
        handles = (ctypes.c_void_p * len(self.scenes))(*[s._h.value for s in self.scenes])
        o = self.options.c()
        self._h = ctypes.c_void_p()
        check(lib.aniso_b200_batch_create(handles, len(self.scenes), _ptr(self.view_scene), len(self.view_scene),
                                          ctypes.byref(o), ctypes.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.aniso_b200_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render_device(self, cameras, rgb_device_ptrs, stream_ptr: int = 0):
        """Enqueues every view (camera k into device buffer rgb_device_ptrs[k]); no wait."""
        if len(cameras) != len(self.view_scene) or len(rgb_device_ptrs) != len(self.view_scene):
            raise ValueError("one camera and one output buffer per view")
        cams = c_cameras(cameras)
        ptrs = (ctypes.c_void_p * len(rgb_device_ptrs))(*[int(p) for p in rgb_device_ptrs])
        check(lib.aniso_b200_batch_render(self._h, cams, ptrs, ctypes.c_void_p(stream_ptr)))

    def sync(self) -> dict:
        st = _lib.Stats()
        check(lib.aniso_b200_batch_sync(self._h, ctypes.byref(st)))
        return _stats_dict(st)
