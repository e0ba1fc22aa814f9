"""The differentiable path: a torch.autograd.Function over the C ABI's training entry points.

    img = rasterize(means, log_scales, quats, opacity_logits, sh, camera, sh_degree=3)
    loss = ((img - target) ** 2).sum(); loss.backward()
    imgs = rasterize_batch([(means, log_scales, quats, opacity_logits, sh), ...], cameras, view_scene)

The parameters are the raw optimizer tensors of pipeline/train_gsplat.py:85-92 (means, log-scales,
quaternions, opacity logits, SH as (n, 16, 3) = sh0 ++ shN), float32 on one CUDA device; the
activations (exp, sigmoid, normalise) run inside the kernels. The output is the (H, W, 3) float
colour before the 8-bit rounding (unclamped, black background). The backward is the library's
hand-written adjoint (deterministic; no atomics).

PyTorch supplies the device memory and the stream; all arithmetic is in libaniso_b200.so.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check, lib
from .renderer import BatchOptions, RenderOptions, c_camera, c_cameras


class Trainer:
    """The work buffers of one forward and its backward (a C-ABI aniso_b200_trainer)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        check(lib.aniso_b200_trainer_create(ctypes.byref(self._h)))

    def close(self):
        if self._h.value:
            lib.aniso_b200_trainer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_pool: list[Trainer] = []


def _acquire() -> Trainer:
    return _pool.pop() if _pool else Trainer()


def _release(t: Trainer):
    _pool.append(t)


class _Lease:
    """Holds a trainer for one forward until its backward, and gives it back to the pool (not
    destroys it) if the graph is dropped without a backward -- e.g. a forward under no_grad."""

    def __init__(self, trainer: Trainer):
        self.trainer = trainer

    def release(self):
        if self.trainer is not None:
            _release(self.trainer)
            self.trainer = None

    def __del__(self):
        self.release()


def _raw_params(means, log_scales, quats, opacity_logits, sh) -> _lib.RawParams:
    n = means.shape[0]
    k = sh.shape[1]
    deg = {4: 1, 16: 3}.get(k)
    if deg is None:
        raise ValueError("sh must hold 4 or 16 coefficients per channel (pad lower degrees with zeros)")
    for name, t, shape in (("means", means, (n, 3)), ("log_scales", log_scales, (n, 3)), ("quats", quats, (n, 4)),
                           ("opacity_logits", opacity_logits, (n,)), ("sh", sh, (n, k, 3))):
        if tuple(t.shape) != shape or t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("%s must be a contiguous float32 CUDA tensor of shape %s" % (name, shape))
    return _lib.RawParams(means.data_ptr(), log_scales.data_ptr(), quats.data_ptr(), opacity_logits.data_ptr(),
                          sh.data_ptr(), n, deg)


class RasterizeFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, log_scales, quats, opacity_logits, sh, camera, options, stats=None):
        means, log_scales, quats = means.contiguous(), log_scales.contiguous(), quats.contiguous()
        opacity_logits, sh = opacity_logits.contiguous(), sh.contiguous()
        params = _raw_params(means, log_scales, quats, opacity_logits, sh)
        img = torch.empty(camera.height, camera.width, 3, dtype=torch.float32, device=means.device)
        trainer = _acquire()
        stream = torch.cuda.current_stream(means.device).cuda_stream
        try:
            check(lib.aniso_b200_train_forward(trainer._h, ctypes.byref(params), ctypes.byref(c_camera(camera)),
                                               ctypes.byref(options.c()), ctypes.c_void_p(img.data_ptr()),
                                               ctypes.c_void_p(stream)))
        except Exception:
            _release(trainer)
            raise
        # The next forward on this trainer is ordered after this one's kernels (same stream).
        ctx.lease = _Lease(trainer)
        if not any(ctx.needs_input_grad[:5]):
            ctx.lease.release()
        ctx.stats = stats
        ctx.save_for_backward(means, log_scales, quats, opacity_logits, sh)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        means, log_scales, quats, opacity_logits, sh = ctx.saved_tensors
        # Fresh zeroed buffers: the backward stores into them without reading them (fresh = 1).
        grads = [torch.zeros_like(t) for t in (means, log_scales, quats, opacity_logits, sh)]
        extra = [ctx.stats[0].data_ptr(), ctx.stats[1].data_ptr()] if ctx.stats is not None else [None, None]
        g = _lib.RawGrads(*[t.data_ptr() for t in grads], *extra, 1)
        gi = grad_img.contiguous().float()
        stream = torch.cuda.current_stream(means.device).cuda_stream
        if ctx.lease.trainer is None:
            raise RuntimeError("this render's backward already ran (its work buffers are reused): render again")
        try:
            check(lib.aniso_b200_train_backward(ctx.lease.trainer._h, ctypes.c_void_p(gi.data_ptr()),
                                                ctypes.byref(g), ctypes.c_void_p(stream)))
        finally:
            # The next forward on this trainer is ordered after the backward's kernels (same stream).
            ctx.lease.release()
        return (*grads, None, None, None)


def rasterize(means, log_scales, quats, opacity_logits, sh, camera, sh_degree: int = 3, splat_scale: float = 1.0,
              stats=None):
    """Differentiable render of one view: (H, W, 3) float32 colour.

    stats: optional (grad2d, visible) float32 CUDA tensors of shape (n,); the backward adds to them
    each Gaussian's |dL/d(screen position)| in NDC units and 1 where it was visible -- what a
    densification strategy accumulates."""
    if stats is not None:
        n = means.shape[0]
        for t in stats:
            if tuple(t.shape) != (n,) or t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
                raise ValueError("stats must be two contiguous float32 CUDA tensors of shape (n,)")
    return RasterizeFunction.apply(means, log_scales, quats, opacity_logits, sh, camera,
                                   RenderOptions(sh_degree, splat_scale), stats)


class RasterizeBatchFunction(torch.autograd.Function):
    """Views of several scenes in one forward and one backward (aniso_b200_train_batch_*)."""

    @staticmethod
    def forward(ctx, meta, *tensors):
        cameras, view_scene, options = meta
        S = len(tensors) // 5
        tensors = [t.contiguous() for t in tensors]
        params = (_lib.RawParams * S)(*[_raw_params(*tensors[5 * s:5 * s + 5]) for s in range(S)])
        device = tensors[0].device
        imgs = [torch.empty(c.height, c.width, 3, dtype=torch.float32, device=device) for c in cameras]
        vs = (ctypes.c_int32 * len(view_scene))(*view_scene)
        cams = c_cameras(cameras)
        ptrs = (ctypes.c_void_p * len(imgs))(*[t.data_ptr() for t in imgs])
        stream = torch.cuda.current_stream(device).cuda_stream
        trainer = _acquire()
        try:
            check(lib.aniso_b200_train_batch_forward(trainer._h, params, S, vs, cams, len(cameras),
                                                     ctypes.byref(options.c()), ptrs, ctypes.c_void_p(stream)))
        except Exception:
            _release(trainer)
            raise
        ctx.lease = _Lease(trainer)
        if not any(ctx.needs_input_grad[1:]):
            ctx.lease.release()
        ctx.n_scenes = S
        ctx.save_for_backward(*tensors)
        return tuple(imgs)

    @staticmethod
    def backward(ctx, *grad_imgs):
        tensors = ctx.saved_tensors
        S = ctx.n_scenes
        # Fresh zeroed buffers: each scene's first view stores without reading them (fresh = 1).
        grads = [torch.zeros_like(t) for t in tensors]
        g = (_lib.RawGrads * S)(*[_lib.RawGrads(*[t.data_ptr() for t in grads[5 * s:5 * s + 5]], None, None, 1)
                                  for s in range(S)])
        # Views outside the loss arrive as zero images (autograd materialises unused outputs' grads).
        gi = [gimg.contiguous().float() for gimg in grad_imgs]
        ptrs = (ctypes.c_void_p * len(gi))(*[t.data_ptr() for t in gi])
        stream = torch.cuda.current_stream(tensors[0].device).cuda_stream
        if ctx.lease.trainer is None:
            raise RuntimeError("this render's backward already ran (its work buffers are reused): render again")
        try:
            check(lib.aniso_b200_train_batch_backward(ctx.lease.trainer._h, ptrs, g, ctypes.c_void_p(stream)))
        finally:
            ctx.lease.release()
        return (None, *grads)


def rasterize_batch(scenes, cameras, view_scene, sh_degree: int = 3, splat_scale: float = 1.0,
                    tile: tuple[int, int] = (16, 16), blend_batch: int = 256, use_graph: bool = True,
                    options: BatchOptions | None = None):
    """Differentiable render of many views of several scenes in one forward/backward.

    scenes: a list of (means, log_scales, quats, opacity_logits, sh) tuples; view k shows scene
    view_scene[k] (the views of a scene consecutive). Returns one (H, W, 3) image per view. The
    gradient of a scene is the sum over its views, added in view order (deterministic).
    options: a launch shape (autotune.tune_train's choice) instead of sh_degree .. use_graph. With
    use_graph, the forward's and the backward's launch sequences are recorded as CUDA graphs on
    the first step of a shape and replayed on the next ones (the parameter, image and gradient
    tensors may move between steps; a new shape or size records again).
    """
    flat = [t for s in scenes for t in s]
    opts = options if options is not None else BatchOptions(sh_degree, splat_scale, tuple(tile), blend_batch,
                                                            use_graph)
    return RasterizeBatchFunction.apply((list(cameras), [int(v) for v in view_scene], opts), *flat)
