"""ORACLE -- test infrastructure, not product code.

Gradient checks of the differentiable path against the FP64 oracle at full size (BigFrame), used
by tests/test_gradients_config3.py and by bench.py's checker leg (outside any timed region), never
by the product:

* fd_check: FP64 central differences (h = 1e-4) of the whole-image L2 loss on randomly sampled raw
  parameters of visible Gaussians, stratified over the five parameter groups. A draw whose two
  evaluations (+h, -h) take different branches of the renderer -- the loss is then not smooth on
  [-h, h] and the difference measures a jump, not a derivative -- is redrawn and counted.
* window_check: the FP64 adjoint of the loss restricted to a pixel window, every raw-parameter
  gradient of every Gaussian, against the same gradients from the GPU.

Relative error of a group: ||g_gpu - g_ref||_2 / ||g_ref||_2 over its entries.
"""
from __future__ import annotations

import numpy as np

GROUPS = ("means", "log_scales", "quats", "opacity_logits", "sh")
GROUP_SIZES = (3, 3, 4, 1, 48)


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def raw_param_arrays(raw):
    """The optimizer's five raw tensors of a RawScene (SH as n x 16 x 3, [coefficient][channel])."""
    n = raw.n
    k = raw.f_rest.shape[1] // 3
    sh = np.concatenate([raw.f_dc.reshape(n, 1, 3), raw.f_rest.reshape(n, 3, k).transpose(0, 2, 1)], 1)
    return [np.ascontiguousarray(a, np.float32) for a in (raw.xyz, raw.scale, raw.rot, raw.opacity, sh)]


def fd_check(big, target, grads, live, samples=256, step=1e-4, seed=2, max_draws=2048):
    """grads: the GPU gradients (five arrays, the raw tensors' shapes) of the whole-image loss
    sum((image - target)^2); live: indices of Gaussians that contribute to the image. Returns per
    group {samples, redrawn, rel_err} and the totals."""
    rng = np.random.default_rng(seed)
    quota = [samples // 5 + (1 if g < samples % 5 else 0) for g in range(5)]
    got = {name: ([], []) for name in GROUPS}
    redrawn = {name: 0 for name in GROUPS}
    pixels = 0
    draws = 0
    for g, name in enumerate(GROUPS):
        size = int(np.prod(grads[g].shape[1:])) if grads[g].ndim > 1 else 1
        while len(got[name][1]) < quota[g]:
            draws += 1
            if draws > max_draws:
                raise RuntimeError("too many discontinuous draws: %s" % redrawn)
            i = int(live[rng.integers(len(live))])
            comp = int(rng.integers(size))
            fd, smooth, px = big.fd(target, i, g, comp, step)
            pixels += px
            if not smooth:
                redrawn[name] += 1
                continue
            gpu = grads[g].reshape(grads[g].shape[0], -1)[i, comp]
            got[name][0].append(float(gpu))
            got[name][1].append(fd)
    out = {name: {"samples": len(got[name][1]), "redrawn": redrawn[name],
                  "rel_err": rel(got[name][0], got[name][1])} for name in GROUPS}
    out["_totals"] = {"samples": sum(quota), "redrawn": sum(redrawn.values()), "step": step,
                      "pixels_evaluated": pixels}
    return out


def window_check(big, x0, y0, grad_window, gpu_grads):
    """gpu_grads: the GPU gradients of the loss whose colour gradient is grad_window on the window
    [x0, x0 + w) x [y0, y0 + h) and zero elsewhere; compared with the FP64 adjoint of that loss."""
    ref = big.adjoint(x0, y0, grad_window)
    out = {}
    for name, a, b in zip(GROUPS, gpu_grads, ref):
        nz = int(np.count_nonzero(np.abs(b.reshape(b.shape[0], -1)).sum(1)))
        out[name] = {"rel_err": rel(a, b), "gaussians": nz}
    return out
