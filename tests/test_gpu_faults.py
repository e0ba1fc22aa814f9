"""Hostile inputs on the GPU path, injected on the host (bad values in the inputs; nothing here
makes the device fault or wait): non-finite means, log-scales and opacity logits, zero and NaN
quaternions, overflowing scales, empty, tiny and oversized cameras, extreme splat scales. Each case
either renders the image the reference CPU renderer (render.cpp) renders from the same activated
inputs, within the image bars, or is refused with a documented status code; the bytes around
every output buffer stay untouched (needs a GPU).

Inputs the reference leaves to undefined behaviour are given one defined meaning here: a Gaussian
whose projection is not finite, or whose radius is a billion pixels or more, is culled -- the
image render.cpp produces on x86-64, where such a splat's float-to-int tile bounds come out empty
(render.cpp:84-89, 159-171). NaN SH coefficients are outside the defined inputs: the reference's
8-bit quantisation of a NaN colour is itself undefined.
"""
import numpy as np
import pytest

import kat
import oracle
from aniso_b200 import scenes

pytestmark = pytest.mark.gpu

GUARD = 64
FILL = 0xAB


@pytest.fixture(scope="module")
def ab():
    import aniso_b200

    assert aniso_b200.GpuRenderer.available()
    return aniso_b200


def cpu_render(gauss, sh, cam, sh_degree=3, splat_scale=1.0):
    if oracle.ReferenceCPU.available():
        return oracle.ReferenceCPU().render(gauss, sh, 3, cam, sh_degree, splat_scale)[0]
    return oracle.Restatement().render(gauss, sh, 3, cam, sh_degree, splat_scale)[0]


def assert_parity(gpu, cpu, what):
    d = int(np.abs(gpu.astype(np.int32) - cpu.astype(np.int32)).max()) if gpu.size else 0
    p = oracle.psnr(gpu, cpu)
    assert d <= 2 and p >= 75.0, "%s: max-abs %d/255, PSNR %.1f dB" % (what, d, p)


POISON = {  # raw-column edits of Gaussians placed in the middle of the view
    "nan_mean": ("xyz", (0,), np.nan),
    "inf_depth": ("xyz", (2,), np.inf),
    "neg_inf_mean": ("xyz", (0,), -np.inf),
    "nan_log_scale": ("scale", (1,), np.nan),
    "inf_log_scale": ("scale", (0,), np.inf),
    "neg_inf_log_scale": ("scale", (2,), -np.inf),    # scale 0: a finite, point-like splat
    "overflow_log_scale": ("scale", (0, 1, 2), 60.0),  # exp(60): the covariance overflows
    "nan_logit": ("opacity", (), np.nan),             # opacity NaN: alpha is 0.99 wherever it reaches
    "inf_logit": ("opacity", (), np.inf),             # opacity 1
    "neg_inf_logit": ("opacity", (), -np.inf),        # opacity 0
    "zero_quat": ("rot", (0, 1, 2, 3), 0.0),          # the identity rotation (ply_loader.cpp:130)
    "nan_quat": ("rot", (0,), np.nan),                # the identity rotation too
}


def poisoned_raw(seed=31):
    raw = scenes.make_raw_scene(3000, (-1.5, -1.0, 3.0), (1.5, 1.0, 7.0), seed)
    raw.scale[:] += 1.0  # a little larger than the generator's, so the poisoned ones would show
    rng = np.random.default_rng(seed)
    for k, (name, (field, cols, value)) in enumerate(sorted(POISON.items())):
        i = 100 + 7 * k
        raw.xyz[i] = (rng.uniform(-0.5, 0.5), rng.uniform(-0.3, 0.3), 4.0)
        arr = getattr(raw, field)
        if cols:
            arr[i, list(cols)] = value
        else:
            arr[i] = value
    return raw


def test_poisoned_scene_matches_cpu_on_every_ingest_path(ab, tmp_path):
    raw = poisoned_raw()
    gauss, sh = oracle.Restatement().activate(raw)  # the reference loader's activation, on the host
    cam = kat.gpu_test_camera(320, 240)
    want = cpu_render(gauss, sh, cam)
    assert want.any()
    host = ab.GpuRenderer(gauss, sh, 3).render(cam)
    assert_parity(host, want, "activated upload")
    raw_dev = ab.GpuRenderer.from_raw(raw).render(cam)  # activated on the device
    assert_parity(raw_dev, want, "raw upload")
    scenes.write_ply(str(tmp_path / "poisoned.ply"), raw)
    ply = ab.GpuRenderer.from_ply(str(tmp_path / "poisoned.ply")).render(cam)
    assert_parity(ply, want, "device PLY ingest")


def test_each_poison_alone(ab):
    """One poisoned Gaussian over a clean background per case: the same image as render.cpp."""
    base = scenes.make_raw_scene(1500, (-1.5, -1.0, 3.0), (1.5, 1.0, 7.0), 33)
    cam = kat.gpu_test_camera(256, 192)
    R = oracle.Restatement()
    for name, (field, cols, value) in sorted(POISON.items()):
        raw = scenes.RawScene(*(np.array(a) for a in (base.xyz, base.f_dc, base.f_rest, base.opacity, base.scale,
                                                      base.rot)))
        raw.xyz[0] = (0.0, 0.0, 4.0)
        raw.scale[0] = (-2.0, -2.0, -2.0)
        raw.opacity[0] = 3.0
        arr = getattr(raw, field)
        if cols:
            arr[0, list(cols)] = value
        else:
            arr[0] = value
        gauss, sh = R.activate(raw)
        assert_parity(ab.GpuRenderer(gauss, sh, 3).render(cam), cpu_render(gauss, sh, cam), name)


def test_culled_poisons_have_zero_finite_gradients(ab):
    """In the differentiable path a Gaussian with a non-finite projection is culled: the image is
    the clean scene's and its gradients are zero, everyone else's finite."""
    import torch

    from aniso_b200.autograd import rasterize
    from oracle import gradcheck

    raw = scenes.make_raw_scene(2000, (-1.5, -1.0, 3.0), (1.5, 1.0, 7.0), 35)
    raw.scale[:] += 1.0
    bad = {"nan_mean": ("xyz", 0), "inf_depth": ("xyz", 2), "nan_log_scale": ("scale", 1),
           "inf_log_scale": ("scale", 0)}
    clean = gradcheck.raw_param_arrays(raw)
    cam = kat.gpu_test_camera(200, 150)
    for k, (name, (field, col)) in enumerate(sorted(bad.items())):
        i = 10 + k
        getattr(raw, field)[i, col] = np.nan if "nan" in name else np.inf
    params = gradcheck.raw_param_arrays(raw)
    ts = [torch.tensor(p, device="cuda", requires_grad=True) for p in params]
    img = rasterize(*ts, cam)
    img.square().sum().backward()
    keep = np.ones(raw.n, bool)
    keep[10:14] = False
    with torch.no_grad():
        ref = rasterize(*[torch.tensor(p[keep], device="cuda") for p in clean], cam)
    np.testing.assert_array_equal(img.detach().cpu().numpy(), ref.cpu().numpy())
    for t in ts:
        g = t.grad.cpu().numpy()
        assert np.isfinite(g).all()
        assert not g[10:14].any()


def guarded_host(shape, pinned=False):
    import torch

    n = int(np.prod(shape))
    buf = torch.full((n + 2 * GUARD,), FILL, dtype=torch.uint8)
    if pinned:
        buf = buf.pin_memory()
    arr = buf.numpy()
    return arr, arr[GUARD:GUARD + n].reshape(shape)


def assert_guards(arr, what):
    assert (arr[:GUARD] == FILL).all() and (arr[-GUARD:] == FILL).all(), what + ": guard band written"


@pytest.mark.parametrize("w,h", [(1, 1), (7, 5), (17, 9), (1283, 719)])
def test_guard_bands_host_and_device(ab, w, h):
    import torch

    raw = poisoned_raw()
    gauss, sh = oracle.Restatement().activate(raw)
    r = ab.GpuRenderer(gauss, sh, 3)
    cam = kat.gpu_test_camera(w, h)
    want = cpu_render(gauss, sh, cam)
    for pinned in (False, True):
        arr, view = guarded_host((h, w, 3), pinned)
        got = r.render(cam, out=view)
        assert_guards(arr, "%dx%d %s" % (w, h, "pinned" if pinned else "pageable"))
        assert_parity(got, want, "%dx%d" % (w, h))
    n = w * h * 3
    dev = torch.full((n + 2 * GUARD,), FILL, dtype=torch.uint8, device="cuda")
    r.render_device(cam, dev.data_ptr() + GUARD, torch.cuda.current_stream().cuda_stream)
    r.sync()
    d = dev.cpu().numpy()
    assert_guards(d, "%dx%d device" % (w, h))
    assert_parity(d[GUARD:GUARD + n].reshape(h, w, 3), want, "%dx%d device" % (w, h))


@pytest.mark.parametrize("w,h", [(0, 240), (320, 0), (-4, 10), (40000, 10), (10, 40000)])
def test_bad_camera_sizes_are_refused(ab, w, h):
    import ctypes

    from aniso_b200 import _lib
    from aniso_b200.renderer import c_camera

    g, sh, deg = kat.random_cloud(500, seed=3)
    r = ab.GpuRenderer(g, sh, deg)
    cam = kat.gpu_test_camera(max(w, 1), max(h, 1))
    cam.width, cam.height = w, h
    arr = np.full(4096, FILL, np.uint8)
    rc = _lib.lib.aniso_b200_render(r._h, ctypes.byref(c_camera(cam)), None,
                                    arr.ctypes.data_as(ctypes.c_void_p), None)
    assert rc == _lib.ERR_ARGUMENT
    assert "camera size" in _lib.last_error()
    assert (arr == FILL).all()
    # the scene is still usable afterwards
    ok = kat.gpu_test_camera(64, 48)
    assert_parity(r.render(ok), cpu_render(g, sh, ok), "after a refused call")


@pytest.mark.parametrize("scale", [0.0, 1e-6, 25.0, 2000.0, float("nan"), float("inf")])
def test_extreme_splat_scales(ab, scale):
    g, sh, deg = kat.random_cloud(3000, seed=5)
    cam = kat.gpu_test_camera(320, 240)
    r = ab.GpuRenderer(g, sh, deg)
    st = {}
    img = r.render(cam, st, options=ab.RenderOptions(splat_scale=scale))
    assert_parity(img, cpu_render(g, sh, cam, splat_scale=scale), "splat_scale %g" % scale)
    if not np.isfinite(scale):
        assert st["tile_pairs"] == 0 and not img.any()
