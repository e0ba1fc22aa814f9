"""ORACLE -- test infrastructure, not product code.

Python handles on the checkers that oracle/Makefile builds:

* :class:`Restatement` -- ``_build/libaniso_oracle.so``, the C restatement (aniso_oracle.c) of the
  reference CPU renderer and of the GPU path's integer work (keys, stable sort, tile ranges).
* :class:`ReferenceCPU` -- ``_ref/libaniso_ref_cpu.so``, the reference's own CPU renderer,
  loader and SH code compiled from its sources (render.cpp, sh.cpp, camera.cpp, ply_loader.cpp).
* :class:`ReferenceGPU` -- ``_ref/libaniso_ref_gpu.so`` (no fast-math: the bit-exact key/range
  oracle) or ``_ref/libaniso_ref_gpu_fast.so`` (as shipped): the reference's own CUDA kernels.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs import this
package, and only as the checker or the timed CPU baseline, never as the product path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "libaniso_oracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libaniso_ref_cpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libaniso_ref_gpu.so")
REF_GPU_FAST_SO = os.path.join(HERE, "_ref", "libaniso_ref_gpu_fast.so")

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int
_F = ctypes.c_float
_U64 = ctypes.c_uint64


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(_P)


def _cam(cam) -> np.ndarray:
    return np.ascontiguousarray(cam.packed(), dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Restatement:
    """The C restatement of the reference path (always buildable: it needs no reference files)."""

    def __init__(self, path: str = RESTATEMENT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " is missing: run `make -C oracle restatement`")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_activate.argtypes = [_I64, _P, _P, _P, _P, _P, _P, _I, _P, _P]
        L.orc_sh_color.argtypes = [_P, _I, _F, _F, _F, _I, _P]
        L.orc_camera_centre.argtypes = [_P, _P]
        L.orc_make_splats.argtypes = [_I64, _P, _P, _I, _P, _I, _I, _I, _F, _P, _P, _P]
        L.orc_render.argtypes = [_I64, _P, _P, _I, _P, _I, _I, _I, _F, _P, _P]
        L.orc_render.restype = _I
        L.orc_sort_keys.argtypes = [_I64, _P, _P, _P, _I, _I, _P, _P, _I64, _P]
        L.orc_sort_keys.restype = _I64
        L.orc_train_forward_f64.argtypes = [_I64, _P, _P, _P, _P, _P, _I, _P, _I, _I, _I, ctypes.c_double, _P]
        L.orc_train_forward_f64.restype = _I
        L.orc_train_backward_f64.argtypes = [_I64, _P, _P, _P, _P, _P, _I, _P, _I, _I, _I, ctypes.c_double, _P,
                                             _P, _P, _P, _P, _P]
        L.orc_train_backward_f64.restype = _I
        L.orc_big_create.argtypes = [_I64, _P, _P, _P, _P, _P, _I, _P, _I, _I, _I, ctypes.c_double]
        L.orc_big_create.restype = _P
        L.orc_big_destroy.argtypes = [_P]
        L.orc_big_counts.argtypes = [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]
        L.orc_big_image.argtypes = [_P, _I, _I, _I, _I, _P]
        L.orc_big_image.restype = _I
        L.orc_big_adjoint.argtypes = [_P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]
        L.orc_big_adjoint.restype = _I
        L.orc_big_fd.argtypes = [_P, _P, _I64, _I, _I, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(_I), ctypes.POINTER(_I64)]
        L.orc_big_fd.restype = _I

    def activate(self, raw):
        n = raw.n
        deg = raw.sh_degree
        k = (deg + 1) ** 2
        gauss = np.empty((n, 11), np.float32)
        sh = np.empty((n, k * 3), np.float32)
        xyz, dc, rest = _f32(raw.xyz), _f32(raw.f_dc), _f32(raw.f_rest)
        op, sc, rot = _f32(raw.opacity), _f32(raw.scale), _f32(raw.rot)
        self.lib.orc_activate(n, _ptr(xyz), _ptr(dc), _ptr(rest), _ptr(op), _ptr(sc), _ptr(rot), deg,
                              _ptr(gauss), _ptr(sh))
        return gauss, sh

    def sh_color(self, sh, scene_degree, d, degree):
        sh = _f32(sh)
        out = np.empty(3, np.float32)
        self.lib.orc_sh_color(_ptr(sh), scene_degree, float(d[0]), float(d[1]), float(d[2]), degree, _ptr(out))
        return out

    def camera_centre(self, cam):
        c = _cam(cam)
        out = np.empty(3, np.float32)
        self.lib.orc_camera_centre(_ptr(c), _ptr(out))
        return out

    def make_splats(self, gauss, sh, scene_degree, cam, sh_degree=3, splat_scale=1.0):
        gauss, sh = _f32(gauss), _f32(sh)
        n = gauss.shape[0]
        out = np.zeros((n, 10), np.float32)
        radius = np.zeros(n, np.int32)
        alive = np.zeros(n, np.uint8)
        c = _cam(cam)
        self.lib.orc_make_splats(n, _ptr(gauss), _ptr(sh), scene_degree, _ptr(c), cam.width, cam.height,
                                 sh_degree, splat_scale, _ptr(out), _ptr(radius), _ptr(alive))
        return out, radius, alive.astype(bool)

    def render(self, gauss, sh, scene_degree, cam, sh_degree=3, splat_scale=1.0):
        gauss, sh = _f32(gauss), _f32(sh)
        img = np.zeros((cam.height, cam.width, 3), np.uint8)
        stats = np.zeros(2, np.int64)
        c = _cam(cam)
        rc = self.lib.orc_render(gauss.shape[0], _ptr(gauss), _ptr(sh), scene_degree, _ptr(c), cam.width,
                                 cam.height, sh_degree, splat_scale, _ptr(img), _ptr(stats))
        if rc != 0:
            raise MemoryError("orc_render failed")
        return img, {"visible": int(stats[0]), "tile_pairs": int(stats[1])}

    def sort_keys(self, tiles_touched, rect, depth, tiles_x, tiles_y):
        """(keys u64[P], values u32[P], ranges u32[T, 2]) as the reference GPU path produces."""
        tt = np.ascontiguousarray(tiles_touched, np.uint32)
        rc = np.ascontiguousarray(rect, np.uint32).reshape(-1, 4)
        dp = _f32(depth)
        total = int(tt.astype(np.int64).sum())
        keys = np.zeros(max(total, 1), np.uint64)
        values = np.zeros(max(total, 1), np.uint32)
        ranges = np.zeros((tiles_x * tiles_y, 2), np.uint32)
        got = self.lib.orc_sort_keys(tt.shape[0], _ptr(tt), _ptr(rc), _ptr(dp), tiles_x, tiles_y, _ptr(keys),
                                     _ptr(values), keys.shape[0], _ptr(ranges))
        assert got == total
        return keys[:total], values[:total], ranges


    # ---- FP64 gradient oracle: raw parameters as float64 arrays (means n x 3, log_scales n x 3,
    # quats n x 4, logits n, sh n x K x 3) ----
    @staticmethod
    def _f64(params):
        return [np.ascontiguousarray(p, dtype=np.float64) for p in params]

    def train_forward_f64(self, params, cam, sh_degree=3, splat_scale=1.0):
        means, ls, q, lg, sh = self._f64(params)
        img = np.zeros((cam.height, cam.width, 3), np.float64)
        c = _cam(cam)
        rc = self.lib.orc_train_forward_f64(means.shape[0], _ptr(means), _ptr(ls), _ptr(q), _ptr(lg), _ptr(sh),
                                            sh.shape[1], _ptr(c), cam.width, cam.height, sh_degree, splat_scale,
                                            _ptr(img))
        assert rc == 0, rc
        return img

    def train_backward_f64(self, params, cam, grad_img, sh_degree=3, splat_scale=1.0):
        means, ls, q, lg, sh = self._f64(params)
        gi = np.ascontiguousarray(grad_img, np.float64)
        grads = [np.zeros_like(a) for a in (means, ls, q, lg, sh)]
        c = _cam(cam)
        rc = self.lib.orc_train_backward_f64(means.shape[0], _ptr(means), _ptr(ls), _ptr(q), _ptr(lg), _ptr(sh),
                                             sh.shape[1], _ptr(c), cam.width, cam.height, sh_degree, splat_scale,
                                             _ptr(gi), *[_ptr(g) for g in grads])
        assert rc == 0, rc
        return grads

    def big_frame(self, params, cam, sh_degree=3, splat_scale=1.0):
        """The FP64 training render of a scene of any size, for local queries (BigFrame)."""
        return BigFrame(self, params, cam, sh_degree, splat_scale)


class BigFrame:
    """FP64 training render (orc_big_*) held for local queries: window images, window adjoints and
    single-parameter central differences of the whole-image L2 loss."""

    GROUPS = ("means", "log_scales", "quats", "opacity_logits", "sh")

    def __init__(self, R: Restatement, params, cam, sh_degree=3, splat_scale=1.0):
        self.R, self.cam = R, cam
        self.params = Restatement._f64(params)  # kept alive: the frame reads them
        means, ls, q, lg, sh = self.params
        c = _cam(cam)
        self.h = R.lib.orc_big_create(means.shape[0], _ptr(means), _ptr(ls), _ptr(q), _ptr(lg), _ptr(sh),
                                      sh.shape[1], _ptr(c), cam.width, cam.height, sh_degree, splat_scale)
        if not self.h:
            raise MemoryError("orc_big_create failed")

    def counts(self):
        v, p = _I64(0), _I64(0)
        self.R.lib.orc_big_counts(self.h, ctypes.byref(v), ctypes.byref(p))
        return v.value, p.value

    def image(self, x0, y0, w, h):
        out = np.zeros((h, w, 3), np.float64)
        assert self.R.lib.orc_big_image(self.h, x0, y0, w, h, _ptr(out)) == 0
        return out

    def adjoint(self, x0, y0, grad):
        grad = np.ascontiguousarray(grad, np.float64)
        h, w = grad.shape[:2]
        grads = [np.zeros_like(a) for a in self.params]
        assert self.R.lib.orc_big_adjoint(self.h, x0, y0, w, h, _ptr(grad), *[_ptr(g) for g in grads]) == 0
        return grads

    def fd(self, target, i, group, comp, step):
        """(central difference, smooth, pixels evaluated) of the whole-image L2 loss vs target."""
        target = np.ascontiguousarray(target, np.float32)
        assert target.shape == (self.cam.height, self.cam.width, 3)
        d, sm, px = ctypes.c_double(0), _I(0), _I64(0)
        assert self.R.lib.orc_big_fd(self.h, _ptr(target), int(i), int(group), int(comp), float(step), ctypes.byref(d),
                                     ctypes.byref(sm), ctypes.byref(px)) == 0
        return d.value, bool(sm.value), px.value

    def close(self):
        if self.h:
            self.R.lib.orc_big_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class ReferenceCPU:
    """The reference CPU renderer, loader and SH code, compiled from the reference's sources."""

    def __init__(self, path: str = REF_CPU_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_cpu_last_error.restype = ctypes.c_char_p
        L.ref_cpu_render.argtypes = [_P, _P, _I64, _I, _P, _I, _I, _I, _F, _P, _P]
        L.ref_cpu_make_splats.argtypes = [_P, _P, _I64, _I, _P, _I, _I, _I, _F, _P, _P, _P]
        L.ref_cpu_sh_color.argtypes = [_P, _I, _F, _F, _F, _I, _P]
        L.ref_cpu_load_ply.argtypes = [ctypes.c_char_p, ctypes.POINTER(_I64), ctypes.POINTER(_I), _P, _P]
        L.ref_cpu_load_colmap.argtypes = [ctypes.c_char_p, ctypes.POINTER(_I), _P]
        L.ref_cpu_camera_centre.argtypes = [_P, _P]
        L.ref_cpu_scene_create.argtypes = [_P, _P, _I64, _I]
        L.ref_cpu_scene_create.restype = _P
        L.ref_cpu_scene_destroy.argtypes = [_P]
        L.ref_cpu_scene_render.argtypes = [_P, _P, _I, _I, _I, _F, _P, _P]

    @staticmethod
    def available(path: str = REF_CPU_SO) -> bool:
        return os.path.exists(path)

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_cpu_last_error().decode())

    def render(self, gauss, sh, scene_degree, cam, sh_degree=3, splat_scale=1.0):
        gauss, sh = _f32(gauss), _f32(sh)
        img = np.zeros((cam.height, cam.width, 3), np.uint8)
        stats = np.zeros(5, np.float64)
        c = _cam(cam)
        self._check(self.lib.ref_cpu_render(_ptr(gauss), _ptr(sh), gauss.shape[0], scene_degree, _ptr(c),
                                            cam.width, cam.height, sh_degree, splat_scale, _ptr(img), _ptr(stats)))
        return img, {"visible": int(stats[0]), "tile_pairs": int(stats[1]), "project_ms": stats[2],
                     "sort_ms": stats[3], "blend_ms": stats[4]}

    def scene(self, gauss, sh, scene_degree):
        """An aniso::Scene built once (as the reference CLI builds it) for repeated renders."""
        return ReferenceCPUScene(self, gauss, sh, scene_degree)

    def make_splats(self, gauss, sh, scene_degree, cam, sh_degree=3, splat_scale=1.0):
        gauss, sh = _f32(gauss), _f32(sh)
        n = gauss.shape[0]
        out = np.zeros((n, 10), np.float32)
        radius = np.zeros(n, np.int32)
        alive = np.zeros(n, np.uint8)
        c = _cam(cam)
        self._check(self.lib.ref_cpu_make_splats(_ptr(gauss), _ptr(sh), n, scene_degree, _ptr(c), cam.width,
                                                 cam.height, sh_degree, splat_scale, _ptr(out), _ptr(radius),
                                                 _ptr(alive)))
        return out, radius, alive.astype(bool)

    def sh_color(self, sh, scene_degree, d, degree):
        sh = _f32(sh)
        out = np.empty(3, np.float32)
        self.lib.ref_cpu_sh_color(_ptr(sh), scene_degree, float(d[0]), float(d[1]), float(d[2]), degree, _ptr(out))
        return out

    def load_ply(self, path):
        n, deg = _I64(0), _I(0)
        self._check(self.lib.ref_cpu_load_ply(path.encode(), ctypes.byref(n), ctypes.byref(deg), None, None))
        gauss = np.zeros((n.value, 11), np.float32)
        sh = np.zeros((n.value, (deg.value + 1) ** 2 * 3), np.float32)
        self._check(self.lib.ref_cpu_load_ply(path.encode(), ctypes.byref(n), ctypes.byref(deg), _ptr(gauss),
                                              _ptr(sh)))
        return gauss, sh, deg.value

    def load_colmap(self, folder):
        count = _I(0)
        self._check(self.lib.ref_cpu_load_colmap(folder.encode(), ctypes.byref(count), None))
        out = np.zeros((count.value, 20), np.float64)
        self._check(self.lib.ref_cpu_load_colmap(folder.encode(), ctypes.byref(count), _ptr(out)))
        return out

    def camera_centre(self, cam):
        c = _cam(cam)
        out = np.empty(3, np.float32)
        self.lib.ref_cpu_camera_centre(_ptr(c), _ptr(out))
        return out


class ReferenceCPUScene:
    """A scene held by the reference CPU library: render() times aniso::render alone."""

    def __init__(self, ref: ReferenceCPU, gauss, sh, scene_degree):
        self.ref = ref
        gauss, sh = _f32(gauss), _f32(sh)
        self.handle = ref.lib.ref_cpu_scene_create(_ptr(gauss), _ptr(sh), gauss.shape[0], scene_degree)
        if not self.handle:
            raise RuntimeError(ref.lib.ref_cpu_last_error().decode())

    def render(self, cam, sh_degree=3, splat_scale=1.0, out=None):
        img = out if out is not None else np.zeros((cam.height, cam.width, 3), np.uint8)
        stats = np.zeros(5, np.float64)
        c = _cam(cam)
        self.ref._check(self.ref.lib.ref_cpu_scene_render(self.handle, _ptr(c), cam.width, cam.height, sh_degree,
                                                          splat_scale, _ptr(img), _ptr(stats)))
        return img, {"visible": int(stats[0]), "tile_pairs": int(stats[1]), "project_ms": stats[2],
                     "sort_ms": stats[3], "blend_ms": stats[4]}

    def close(self):
        if self.handle:
            self.ref.lib.ref_cpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


class ReferenceGPU:
    """The reference's CUDA kernels (gpu_render.cu) driven stage by stage; device pointers are
    passed as integers (e.g. torch ``tensor.data_ptr()``)."""

    def __init__(self, fast_math: bool = False):
        path = REF_GPU_FAST_SO if fast_math else REF_GPU_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.refgpu_last_error.restype = ctypes.c_char_p
        L.refgpu_preprocess.argtypes = [_I, _U64, _U64, _U64, _U64, _U64, _I, _P, _I, _I, _I, _F,
                                        _U64, _U64, _U64, _U64, _U64, _U64]
        L.refgpu_sort.argtypes = [_I, _U64, _U64, _U64, _I, _I, _U64, _U64, _U64, _U64, ctypes.POINTER(_U64)]
        L.refgpu_blend.argtypes = [_U64, _U64, _U64, _U64, _U64, _I, _I, _U64]
        L.refgpu_renderer_create.argtypes = [_P, _P, _I64, _I]
        L.refgpu_renderer_create.restype = _P
        L.refgpu_renderer_render.argtypes = [_P, _P, _I, _I, _I, _F, _P, _P]
        L.refgpu_renderer_destroy.argtypes = [_P]

    @staticmethod
    def available(fast_math: bool = False) -> bool:
        return os.path.exists(REF_GPU_FAST_SO if fast_math else REF_GPU_SO)

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.refgpu_last_error().decode())

    def preprocess(self, n, pos, scale, rot, opacity, sh, scene_degree, cam, sh_degree, splat_scale,
                   uv, conic_opacity, depth, rgb, rect, tiles_touched):
        c = _cam(cam)
        self._check(self.lib.refgpu_preprocess(n, pos, scale, rot, opacity, sh, scene_degree, _ptr(c), cam.width,
                                               cam.height, sh_degree, splat_scale, uv, conic_opacity, depth, rgb,
                                               rect, tiles_touched))

    def sort(self, n, tiles_touched, rect, depth, tiles_x, tiles_y, keys_out, values_out, capacity, ranges_out):
        total = _U64(0)
        self._check(self.lib.refgpu_sort(n, tiles_touched, rect, depth, tiles_x, tiles_y, keys_out, values_out,
                                         capacity, ranges_out, ctypes.byref(total)))
        return int(total.value)

    def blend(self, ranges, values, uv, conic_opacity, rgb, w, h, out):
        self._check(self.lib.refgpu_blend(ranges, values, uv, conic_opacity, rgb, w, h, out))

    def renderer(self, gauss, sh, degree):
        gauss, sh = _f32(gauss), _f32(sh)
        h = self.lib.refgpu_renderer_create(_ptr(gauss), _ptr(sh), gauss.shape[0], degree)
        if not h:
            raise RuntimeError(self.lib.refgpu_last_error().decode())
        return h

    def render(self, handle, cam, sh_degree=3, splat_scale=1.0):
        img = np.zeros((cam.height, cam.width, 3), np.uint8)
        stats = np.zeros(5, np.float64)
        c = _cam(cam)
        self._check(self.lib.refgpu_renderer_render(handle, _ptr(c), cam.width, cam.height, sh_degree, splat_scale,
                                                    _ptr(img), _ptr(stats)))
        return img, {"visible": int(stats[0]), "tile_pairs": int(stats[1]), "project_ms": stats[2],
                     "sort_ms": stats[3], "blend_ms": stats[4]}

    def destroy(self, handle):
        self.lib.refgpu_renderer_destroy(handle)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """PSNR in dB of two RGB8 images, as tests/test_gpu_render.cpp:28-36 computes it."""
    d = (a.astype(np.float64) - b.astype(np.float64)) / 255.0
    mse = float((d * d).mean()) if d.size else 0.0
    return 1e9 if mse == 0 else 10.0 * np.log10(1.0 / mse)
