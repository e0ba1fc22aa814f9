"""Launch-shape autotuner for batched rendering.

For a batch (its scenes and its cameras), times every candidate launch shape -- tile shape
(8x8, 16x16, 16x32), blend batch (128, 256 splats staged per round), widest radix digit of the
tile sort (8 or 9 bits; 9 saves a pass when the batch's tiles need 9, 17-18 or 25-27 key bits) --
with the batch's own CUDA graph, keeps the fastest, and caches the choice in a JSON file keyed by
the GPU name and a signature of the workload (Gaussian counts, view count, resolutions). Every candidate renders the
same image (the tile shape only changes how pixels are grouped, the digit width how many passes the
sort takes), so the choice is a pure speed decision; the tuner checks that the candidates agree on one view before it trusts them.

    best = tune(scenes, view_scene, cameras)            # -> BatchOptions
    batch = BatchRenderer(scenes, view_scene, best)
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from .renderer import BatchOptions, BatchRenderer

TILES = [(8, 8), (16, 16), (16, 32)]
BLEND_BATCHES = [128, 256]
RADIX_BITS = [8, 9]
CACHE_PATH = os.path.join(os.path.expanduser("~"), ".cache", "aniso_b200", "autotune.json")
# Largest norm-wise relative difference of two launch shapes' gradients of one tensor.
GRAD_RTOL = 1e-4


def grad_rel_diff(a, b) -> float:
    """|a - b| / |b| in the 2-norm over the whole tensor (0 for two zero tensors)."""
    import torch

    den = float(torch.linalg.vector_norm(b.double()))
    num = float(torch.linalg.vector_norm(a.double() - b.double()))
    return num / den if den > 0 else num


def signature(scenes, view_scene, cameras, sh_degree: int, splat_scale: float) -> str:
    """Workload key: Gaussians per scene, the view -> scene map, resolutions, colour options."""
    parts = [",".join(str(s.n) for s in scenes), ",".join(str(int(v)) for v in view_scene),
             ",".join("%dx%d" % (c.width, c.height) for c in cameras), "sh%d" % sh_degree, "s%g" % splat_scale]
    return hashlib.sha1("|".join(parts).encode()).hexdigest()[:16]


def _load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(path, cache):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only costs a re-tune next time


def time_batch(batch: BatchRenderer, cameras, ptrs, stream, warmup: int = 2, iters: int = 5) -> float:
    """Device milliseconds per batched render (CUDA events on `stream`)."""
    import torch

    from ._lib import AnisoError

    for _ in range(warmup):
        for _attempt in range(3):  # a first frame may overflow the pair capacity and grow it
            batch.render_device(cameras, ptrs, stream.cuda_stream)
            try:
                batch.sync()
                break
            except AnisoError as e:
                if "pair capacity" not in str(e):
                    raise
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(iters):
        batch.render_device(cameras, ptrs, stream.cuda_stream)
    e1.record(stream)
    batch.sync()
    return e0.elapsed_time(e1) / iters


def tune(scenes, view_scene, cameras, sh_degree: int = 3, splat_scale: float = 1.0, use_graph: bool = True,
         cache_path: str | None = CACHE_PATH, force: bool = False, report: list | None = None) -> BatchOptions:
    """The fastest launch shape for this batch (from the cache when it holds this GPU/workload)."""
    import torch

    gpu = torch.cuda.get_device_name()
    key = "%s|%s" % (gpu, signature(scenes, view_scene, cameras, sh_degree, splat_scale))
    cache = _load_cache(cache_path) if cache_path else {}
    if not force and key in cache:
        c = cache[key]
        return BatchOptions(sh_degree, splat_scale, tuple(c["tile"]), int(c["blend_batch"]), use_graph,
                            int(c.get("radix_bits", 8)))

    outs = [torch.empty((c.height, c.width, 3), dtype=torch.uint8, device="cuda") for c in cameras]
    ptrs = [o.data_ptr() for o in outs]
    stream = torch.cuda.Stream()
    results = []
    probe = None
    for tile in TILES:
        for bb in BLEND_BATCHES:
            for bits in RADIX_BITS:
                opt = BatchOptions(sh_degree, splat_scale, tile, bb, use_graph, bits)
                b = BatchRenderer(scenes, view_scene, opt)
                ms = time_batch(b, cameras, ptrs, stream)
                img = outs[0].cpu().numpy()
                if probe is None:
                    probe = img
                elif not np.array_equal(img, probe):
                    raise RuntimeError("launch shapes disagree on the image (tile %s, batch %d, %d-bit digits)"
                                       % (tile, bb, bits))
                results.append({"tile": list(tile), "blend_batch": bb, "radix_bits": bits, "ms": ms})
                b.close()
    best = min(results, key=lambda r: r["ms"])
    if report is not None:
        report.extend(results)
    if cache_path:
        cache[key] = dict(best, candidates=results)
        _store_cache(cache_path, cache)
    return BatchOptions(sh_degree, splat_scale, tuple(best["tile"]), int(best["blend_batch"]), use_graph,
                        int(best["radix_bits"]))


def tune_train(scenes, cameras, view_scene, sh_degree: int = 3, splat_scale: float = 1.0, use_graph: bool = True,
               cache_path: str | None = CACHE_PATH, force: bool = False, report: list | None = None,
               iters: int = 3) -> BatchOptions:
    """The fastest launch shape for a training step of this batch: one batched forward
    (rasterize_batch) and its backward against fixed random upstream gradients, per candidate
    shape, timed with CUDA events; the candidates must agree on every image bit for bit and on the
    gradients to rounding, within GRAD_RTOL norm-wise per tensor (each Gaussian sums one slot per
    tile it touches, so the tile grid groups the same terms differently). scenes: the (means, log_scales, quats, opacity_logits, sh) tensors
    of each scene."""
    import torch

    from .autograd import rasterize_batch

    class _N:  # the signature wants Gaussian counts
        def __init__(self, n):
            self.n = n

    gpu = torch.cuda.get_device_name()
    key = "train|%s|%s" % (gpu, signature([_N(s[0].shape[0]) for s in scenes], view_scene, cameras, sh_degree,
                                          splat_scale))
    cache = _load_cache(cache_path) if cache_path else {}
    if not force and key in cache:
        c = cache[key]
        return BatchOptions(sh_degree, splat_scale, tuple(c["tile"]), int(c["blend_batch"]), use_graph,
                            int(c.get("radix_bits", 8)))
    gen = torch.Generator(device="cuda").manual_seed(4)
    ups = [torch.randn((c.height, c.width, 3), device="cuda", generator=gen) for c in cameras]
    leaves = [[t.detach().requires_grad_(True) for t in s] for s in scenes]

    def step(opt):
        for group in leaves:
            for t in group:
                t.grad = None
        imgs = rasterize_batch(leaves, cameras, view_scene, options=opt)
        torch.autograd.backward(imgs, ups)
        return imgs

    results, probe = [], None
    for tile in TILES:
        for bb in BLEND_BATCHES:
            for bits in RADIX_BITS:
                opt = BatchOptions(sh_degree, splat_scale, tile, bb, use_graph, bits)
                imgs = step(opt)  # also records the graphs and sizes the buffers
                got = ([i.detach().clone() for i in imgs], [t.grad.clone() for g in leaves for t in g])
                if probe is None:
                    probe = got
                else:
                    # Images agree bit for bit; the gradients are the same sums grouped by another
                    # tile grid, so they agree to rounding: per tensor, the norm of the difference
                    # within GRAD_RTOL of the norm (single entries that are sums of many terms of
                    # both signs can differ relatively more).
                    if not all(torch.equal(a, b) for a, b in zip(got[0], probe[0])):
                        raise RuntimeError("launch shapes disagree on an image (tile %s, batch %d, %d-bit digits)"
                                           % (tile, bb, bits))
                    worst = max(grad_rel_diff(a, b) for a, b in zip(got[1], probe[1]))
                    if worst > GRAD_RTOL:
                        raise RuntimeError("launch shapes disagree on the gradients by %.3g (tile %s, batch %d, "
                                           "%d-bit digits)" % (worst, tile, bb, bits))
                step(opt)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for _ in range(iters):
                    step(opt)
                e1.record()
                torch.cuda.synchronize()
                results.append({"tile": list(tile), "blend_batch": bb, "radix_bits": bits,
                                "ms": e0.elapsed_time(e1) / iters})
    best = min(results, key=lambda r: r["ms"])
    if report is not None:
        report.extend(results)
    if cache_path:
        cache[key] = dict(best, candidates=results)
        _store_cache(cache_path, cache)
    return BatchOptions(sh_degree, splat_scale, tuple(best["tile"]), int(best["blend_batch"]), use_graph,
                        int(best["radix_bits"]))


__all__ = ["tune", "tune_train", "time_batch", "signature", "grad_rel_diff", "GRAD_RTOL", "TILES", "BLEND_BATCHES",
           "RADIX_BITS", "CACHE_PATH"]
