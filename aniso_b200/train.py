"""A training step around the differentiable rasterizer: the reference's 3DGS loop
(pipeline/train_gsplat.py:138-185) with this library in place of the third-party gsplat.

    model = GaussianModel.from_raw(means, log_scales, quats, opacity_logits, sh, scene_scale)
    trainer = Trainer(model, total_steps=30000)
    loss = trainer.step(camera, target_image)        # render, L1 + SSIM loss, adjoint, Adam, densify

- Loss: 0.8 L1 + 0.2 (1 - SSIM), SSIM with an 11x11 Gaussian window of sigma 1.5 (as the reference).
- Optimizer: Adam with the reference's per-group learning rates and eps = 1e-15; the means' rate
  decays exponentially to 1% over the run (its ExponentialLR); one fused launch for all groups
  (aniso_b200_adam_step).
- Densification: the published rules of gsplat's DefaultStrategy (gsplat 1.5.3, the version the
  reference pins, pipeline/setup_toolchain.py:95), restated here: accumulate each Gaussian's
  screen-space gradient norm (NDC units) over the steps it is visible; every `refine_every` steps
  between `refine_start` and `refine_stop`, duplicate the small ones whose mean norm exceeds
  `grow_grad2d`, split the large ones in two (positions sampled from the Gaussian, scales / 1.6),
  prune the nearly transparent and, after the first opacity reset, the too large; every
  `reset_every` steps clamp the opacities to twice the pruning threshold. New entries start with
  zero Adam moments, as gsplat's operations leave them.

PyTorch holds the tensors and does the bookkeeping (concatenation, masks, the SSIM convolution); the
rendering, the adjoint and the optimizer update are this library's kernels.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import torch
import torch.nn.functional as F

from . import _lib
from ._lib import check, lib
from .autograd import rasterize

NAMES = ("means", "log_scales", "quats", "opacity_logits", "sh")


@dataclasses.dataclass
class Densify:
    """gsplat DefaultStrategy's defaults."""

    prune_opa: float = 0.005
    grow_grad2d: float = 0.0002
    grow_scale3d: float = 0.01
    prune_scale3d: float = 0.1
    refine_start: int = 500
    refine_stop: int = 15000
    reset_every: int = 3000
    refine_every: int = 100


class GaussianModel:
    """The optimizer's raw tensors (train_gsplat.py:85-92 layout; SH as (n, 16, 3)) and Adam state."""

    def __init__(self, params: dict, scene_scale: float):
        self.p = {k: params[k].detach().contiguous().float().requires_grad_(True) for k in NAMES}
        self.scene_scale = float(scene_scale)
        self.m = {k: torch.zeros_like(self.p[k]) for k in NAMES}
        self.v = {k: torch.zeros_like(self.p[k]) for k in NAMES}
        n = self.n
        self.grad2d = torch.zeros(n, device=self.device)
        self.visible = torch.zeros(n, device=self.device)

    @classmethod
    def from_raw(cls, means, log_scales, quats, opacity_logits, sh, scene_scale: float):
        return cls(dict(zip(NAMES, (means, log_scales, quats, opacity_logits, sh))), scene_scale)

    @property
    def n(self) -> int:
        return int(self.p["means"].shape[0])

    @property
    def device(self):
        return self.p["means"].device

    def tensors(self):
        return [self.p[k] for k in NAMES]

    # ---- structural edits (new entries get zero moments, as gsplat's ops do) ----------------------
    def _replace(self, keep: torch.Tensor, new: dict):
        for k in NAMES:
            old = self.p[k].detach()
            self.p[k] = torch.cat([old[keep], new[k]]).contiguous().requires_grad_(True)
            for st in (self.m, self.v):
                st[k] = torch.cat([st[k][keep], torch.zeros_like(new[k])]).contiguous()
        count = int(new["means"].shape[0])
        self.grad2d = torch.cat([self.grad2d[keep], torch.zeros(count, device=self.device)])
        self.visible = torch.cat([self.visible[keep], torch.zeros(count, device=self.device)])

    def duplicate(self, mask: torch.Tensor):
        keep = torch.ones(self.n, dtype=torch.bool, device=self.device)
        self._replace(keep, {k: self.p[k].detach()[mask] for k in NAMES})

    def split(self, mask: torch.Tensor, generator=None):
        """Each selected Gaussian becomes two: centres sampled from it, scales divided by 1.6."""
        sel = {k: self.p[k].detach()[mask] for k in NAMES}
        scales = torch.exp(sel["log_scales"])
        q = F.normalize(sel["quats"], dim=-1)
        w, x, y, z = q.unbind(-1)
        R = torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                         2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                         2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1).view(-1, 3, 3)
        noise = torch.randn((2,) + scales.shape, device=self.device, generator=generator)
        offsets = torch.einsum("nij,bnj->bni", R, scales[None] * noise)
        new = {"means": (sel["means"][None] + offsets).reshape(-1, 3),
               "log_scales": torch.log(scales / 1.6).repeat(2, 1)}
        for k in ("quats", "opacity_logits", "sh"):
            new[k] = sel[k].repeat((2,) + (1,) * (sel[k].dim() - 1))
        self._replace(~mask, new)

    def prune(self, mask: torch.Tensor):
        self._replace(~mask, {k: self.p[k].detach()[:0] for k in NAMES})


def _gauss_window(size=11, sigma=1.5, device=None):
    g = torch.exp(-((torch.arange(size, device=device) - size // 2) ** 2).float() / (2 * sigma * sigma))
    g = g / g.sum()
    return (g[:, None] * g[None, :])[None, None].repeat(3, 1, 1, 1)


def ssim(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Mean SSIM of two (H, W, 3) images in [0, 1] (11x11 Gaussian window, sigma 1.5)."""
    x, y = a.permute(2, 0, 1)[None], b.permute(2, 0, 1)[None]
    w = _gauss_window(device=a.device)
    mu_x, mu_y = F.conv2d(x, w, groups=3), F.conv2d(y, w, groups=3)
    sxx = F.conv2d(x * x, w, groups=3) - mu_x ** 2
    syy = F.conv2d(y * y, w, groups=3) - mu_y ** 2
    sxy = F.conv2d(x * y, w, groups=3) - mu_x * mu_y
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    s = ((2 * mu_x * mu_y + c1) * (2 * sxy + c2)) / ((mu_x ** 2 + mu_y ** 2 + c1) * (sxx + syy + c2))
    return s.mean()


def adam_step(model: GaussianModel, lrs: dict, lr_sh_rest: float, step: int, beta1=0.9, beta2=0.999, eps=1e-15):
    """One fused Adam launch over the five tensors (SH coefficient 0 at lrs['sh'], the rest at
    lr_sh_rest), on the current stream."""
    groups = (_lib.AdamGroup * len(NAMES))()
    zero_grads = []  # stand-ins for parameters without a gradient, alive until the launch is enqueued
    for k, name in enumerate(NAMES):
        p = model.p[name]
        g = p.grad if p.grad is not None else torch.zeros_like(p)
        if p.grad is None:
            zero_grads.append(g)
        if name == "sh":
            groups[k] = _lib.AdamGroup(p.data_ptr(), g.data_ptr(), model.m[name].data_ptr(), model.v[name].data_ptr(),
                                       p.numel(), float(lr_sh_rest), float(lrs[name]), 3 * p.shape[1], 3, float(eps))
        else:
            groups[k] = _lib.AdamGroup(p.data_ptr(), g.data_ptr(), model.m[name].data_ptr(), model.v[name].data_ptr(),
                                       p.numel(), float(lrs[name]), 0.0, 0, 0, float(eps))
    stream = torch.cuda.current_stream(model.device).cuda_stream
    check(lib.aniso_b200_adam_step(groups, len(NAMES), int(step), float(beta1), float(beta2),
                                   ctypes.c_void_p(stream)))


class Trainer:
    def __init__(self, model: GaussianModel, total_steps: int = 30000, densify: Densify | None = None,
                 sh_degree: int = 3, seed: int = 0):
        self.model = model
        self.total = int(total_steps)
        self.densify = densify or Densify()
        self.sh_degree = sh_degree
        self.steps = 0
        self.gen = torch.Generator(device=model.device)
        self.gen.manual_seed(seed)
        s = model.scene_scale
        # train_gsplat.py:160-161
        self.lrs = {"means": 1.6e-4 * s, "log_scales": 5e-3, "quats": 1e-3, "opacity_logits": 5e-2, "sh": 2.5e-3}
        self.lr_sh_rest = 2.5e-3 / 20

    def step(self, camera, target: torch.Tensor) -> float:
        """One training step on one view: returns the loss."""
        m, d = self.model, self.densify
        deg = min(self.steps // 1000, self.sh_degree)  # train_gsplat.py:176
        for t in m.tensors():
            t.grad = None
        img = rasterize(*m.tensors(), camera, sh_degree=deg, stats=(m.grad2d, m.visible))
        loss = 0.8 * (img - target).abs().mean() + 0.2 * (1 - ssim(img, target))
        loss.backward()
        lrs = dict(self.lrs)
        lrs["means"] = self.lrs["means"] * (0.01 ** (self.steps / max(self.total, 1)))  # ExponentialLR
        adam_step(m, lrs, self.lr_sh_rest, self.steps + 1)
        self.steps += 1
        self._refine(self.steps)
        return float(loss.detach())

    def _refine(self, step: int):
        m, d = self.model, self.densify
        if step >= d.refine_stop:
            return
        if step > d.refine_start and step % d.refine_every == 0:
            with torch.no_grad():
                grads = m.grad2d / m.visible.clamp_min(1)
                high = grads > d.grow_grad2d
                small = torch.exp(m.p["log_scales"]).max(-1).values <= d.grow_scale3d * m.scene_scale
                m.duplicate(high & small)
                grown = torch.cat([high & ~small, torch.zeros(int((high & small).sum()), dtype=torch.bool,
                                                              device=m.device)])
                m.split(grown, self.gen)
                prune = torch.sigmoid(m.p["opacity_logits"]) < d.prune_opa
                if step > d.reset_every:
                    prune |= torch.exp(m.p["log_scales"]).max(-1).values > d.prune_scale3d * m.scene_scale
                m.prune(prune)
                m.grad2d.zero_()
                m.visible.zero_()
        if step % d.reset_every == 0:
            with torch.no_grad():
                cap = math.log(2 * d.prune_opa / (1 - 2 * d.prune_opa))
                m.p["opacity_logits"].clamp_(max=cap)
                m.m["opacity_logits"].zero_()
                m.v["opacity_logits"].zero_()
