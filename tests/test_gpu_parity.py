"""Parity of the B200 rasterizer with the reference, through the C ABI (needs a GPU).

Bars: images within 2/255 max-abs and at least 75 dB PSNR of the reference CPU
renderer (render.cpp); tile ranges, sorted keys and values bit-identical to the reference GPU
path (gpu_render.cu built without fast-math) given the same projection; the projection itself
bit-identical to the reference preprocess kernel built the same way (depth, uv, conic, opacity,
rectangle, tiles touched and the SH colour).
"""
import functools

import numpy as np
import pytest

import kat
import oracle
from aniso_b200 import scenes

pytestmark = pytest.mark.gpu

MAX_ABS = 2      # levels of 255
MIN_PSNR = 75.0  # dB


@pytest.fixture(scope="module")
def ab():
    import aniso_b200

    assert aniso_b200.GpuRenderer.available(), "no CUDA device"
    return aniso_b200


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def cpu_render(gauss, sh, deg, cam, sh_degree=3, splat_scale=1.0):
    """The reference CPU renderer where it was built, else the bit-identical restatement."""
    if oracle.ReferenceCPU.available():
        return oracle.ReferenceCPU().render(gauss, sh, deg, cam, sh_degree, splat_scale)
    return oracle.Restatement().render(gauss, sh, deg, cam, sh_degree, splat_scale)


def compare(gpu, cpu):
    d = np.abs(gpu.astype(np.int32) - cpu.astype(np.int32))
    return int(d.max()) if d.size else 0, oracle.psnr(gpu, cpu)


def assert_image_parity(gpu, cpu, what=""):
    m, p = compare(gpu, cpu)
    assert m <= MAX_ABS and p >= MIN_PSNR, "%s: max-abs %d/255, PSNR %.1f dB" % (what, m, p)
    return m, p


# ---- the reference's known-answer tests (test_render.cpp:40-73), on the GPU ---------------------

def test_kat_single_gaussian(ab):
    g, sh, deg = kat.kat_single()
    cam = kat.kat_camera()
    img = ab.GpuRenderer(g, sh, deg).render(cam)
    variance = np.float32(3.2) * np.float32(3.2) + np.float32(0.3)
    expected = np.float32(0.8) * np.exp(np.float32(-0.5) * np.float32(0.5) / variance) * np.float32(255.0)
    assert abs(int(img[32, 32, 0]) - int(expected + 0.5)) <= 1
    assert img[32, 32, 1] == 0 and img[2, 2, 0] == 0
    assert_image_parity(img, cpu_render(g, sh, deg, cam)[0], "single")


def test_kat_front_hides_back(ab):
    g, sh, deg = kat.kat_front_back()
    cam = kat.kat_camera()
    img = ab.GpuRenderer(g, sh, deg).render(cam)
    assert img[32, 32, 1] > 240 and img[32, 32, 2] < 10
    assert_image_parity(img, cpu_render(g, sh, deg, cam)[0], "front/back")


def test_kat_behind_camera_is_culled(ab):
    g, sh, deg = kat.kat_behind()
    st = {}
    img = ab.GpuRenderer(g, sh, deg).render(kat.kat_camera(), st)
    assert st["visible"] == 0 and st["tile_pairs"] == 0
    assert not img.any()


# ---- test_gpu_render.cpp:62-91, with the tighter bars -------------------------------------------

@pytest.mark.parametrize("w,h", [(320, 240), (333, 217)])
def test_random_cloud_vs_cpu(ab, w, h):
    g, sh, deg = kat.random_cloud(20000)
    cam = kat.gpu_test_camera(w, h)
    st = {}
    img = ab.GpuRenderer(g, sh, deg).render(cam, st)
    cpu, cst = cpu_render(g, sh, deg, cam)
    assert st["visible"] == cst["visible"]
    assert_image_parity(img, cpu, "%dx%d" % (w, h))


def test_degree0_and_empty_view(ab):
    g, sh, deg = kat.random_cloud(20000)
    r = ab.GpuRenderer(g, sh, deg)
    cam = kat.gpu_test_camera(320, 240)
    opt = ab.RenderOptions(sh_degree=0)
    assert_image_parity(r.render(cam, options=opt), cpu_render(g, sh, deg, cam, sh_degree=0)[0], "degree 0")
    behind = scenes.Camera(320, 240, cam.fx, cam.fy, cam.cx, cam.cy, np.diag([-1.0, 1.0, -1.0]), np.zeros(3))
    st = {}
    black = r.render(behind, st)
    assert not black.any() and st["tile_pairs"] == 0


def test_splat_scale_and_degrees(ab):
    g, sh, deg = kat.random_cloud(5000, seed=11)
    r = ab.GpuRenderer(g, sh, deg)
    cam = kat.gpu_test_camera(256, 192)
    for d, s in [(1, 1.0), (2, 0.5), (3, 1.7)]:
        img = r.render(cam, options=ab.RenderOptions(sh_degree=d, splat_scale=s))
        assert_image_parity(img, cpu_render(g, sh, deg, cam, d, s)[0], "degree %d scale %g" % (d, s))


# ---- bit-exact projection and sort vs the reference GPU kernels (no fast-math) -------------------

def reference_projection(torch, g, sh, deg, cam, sh_degree=3, splat_scale=1.0):
    """Runs the reference preprocess kernel (gpu_render.cu:86-145) on the same activated scene."""
    ref = oracle.ReferenceGPU(fast_math=False)
    n = g.shape[0]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pos, scale = dev(g[:, 0:3]), dev(g[:, 3:6])
    rot, op, shd = dev(g[:, 6:10]), dev(g[:, 10]), dev(sh)
    out = {"uv": torch.zeros(n, 2, device="cuda"), "conic_opacity": torch.zeros(n, 4, device="cuda"),
           "depth": torch.zeros(n, device="cuda"), "rgb": torch.zeros(n, 3, device="cuda"),
           "rect": torch.zeros(n, 4, dtype=torch.int32, device="cuda"),
           "tiles_touched": torch.zeros(n, dtype=torch.int32, device="cuda")}
    ref.preprocess(n, pos.data_ptr(), scale.data_ptr(), rot.data_ptr(), op.data_ptr(), shd.data_ptr(), deg, cam,
                   sh_degree, splat_scale, out["uv"].data_ptr(), out["conic_opacity"].data_ptr(),
                   out["depth"].data_ptr(), out["rgb"].data_ptr(), out["rect"].data_ptr(),
                   out["tiles_touched"].data_ptr())
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["rect"] = res["rect"].view(np.uint32)
    res["tiles_touched"] = res["tiles_touched"].view(np.uint32)
    return res


def reference_sort(torch, proj, tiles_x, tiles_y):
    """Runs the reference's scan, duplicate, CUB sort and tileRanges (gpu_render.cu:324-345)."""
    ref = oracle.ReferenceGPU(fast_math=False)
    n = proj["depth"].shape[0]
    total = int(proj["tiles_touched"].astype(np.int64).sum())
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tt = dev(proj["tiles_touched"].view(np.int32))
    rect = dev(proj["rect"].view(np.int32))
    depth = dev(proj["depth"])
    keys = torch.zeros(max(total, 1), dtype=torch.int64, device="cuda")
    values = torch.zeros(max(total, 1), dtype=torch.int32, device="cuda")
    ranges = torch.zeros(tiles_x * tiles_y, 2, dtype=torch.int32, device="cuda")
    got = ref.sort(n, tt.data_ptr(), rect.data_ptr(), depth.data_ptr(), tiles_x, tiles_y, keys.data_ptr(),
                   values.data_ptr(), max(total, 1), ranges.data_ptr())
    assert got == total
    return (keys.cpu().numpy().view(np.uint64)[:total], values.cpu().numpy().view(np.uint32)[:total],
            ranges.cpu().numpy().view(np.uint32))


@functools.lru_cache(maxsize=1)
def config2_scene():
    """The 740k-Gaussian bench scene, activated on the host as the reference loader does, and its
    16 ring cameras (generated once per test session)."""
    raws, camsets = scenes.config(2)
    return oracle.Restatement().activate(raws[0]) + (3,), camsets[0]


def pushed_cloud(n_far, z_lo, z_hi):
    """The 20k cloud with n_far of its Gaussians moved along their lines of sight to depths in
    [z_lo, z_hi): they stay on screen (and visible: the 0.3-pixel dilation gives every splat in
    front of the camera a few pixels)."""
    g, sh, d = kat.random_cloud(20000)
    g = g.copy()
    rng = np.random.default_rng(5)
    k = rng.choice(len(g), n_far, replace=False)
    z = rng.uniform(z_lo, z_hi, n_far).astype(np.float32)
    ratio = z / g[k, 2]
    g[k, 0] *= ratio
    g[k, 1] *= ratio
    g[k, 2] = z
    return g, sh, d


PROJ_CASES = {
    # at most 4096 tiles: the one-pass tile binning; above: the LSD tile passes and the ranges kernel
    "cloud20k": lambda: (kat.random_cloud(20000), kat.gpu_test_camera(333, 217)),
    # depths up to 8100: three 9-bit depth passes, keys up to the top of their 27 bits
    "cloud20k_deep": lambda: (pushed_cloud(300, 4000.0, 8100.0), kat.gpu_test_camera(333, 217)),
    # depths past 8192: the scene's box keeps the four 8-bit depth passes
    "cloud20k_far": lambda: (pushed_cloud(300, 8000.0, 30000.0), kat.gpu_test_camera(333, 217)),
    "cloud20k_4096tiles": lambda: (kat.random_cloud(20000), kat.gpu_test_camera(1024, 1024)),  # the binning's largest
    "cloud20k_8160tiles": lambda: (kat.random_cloud(20000), kat.gpu_test_camera(1920, 1088)),
    "config1": lambda: ((lambda s: oracle.Restatement().activate(s) + (3,))(scenes.config(1)[0][0]),
                        scenes.config(1)[1][0][0]),
    # the bench workload itself: 740k Gaussians, ~325k visible, ~1.6M pairs at 1280x720
    "config2_ring0": lambda: (config2_scene()[0], config2_scene()[1][0]),
    "config2_ring5": lambda: (config2_scene()[0], config2_scene()[1][5]),
}


@pytest.mark.parametrize("case", sorted(PROJ_CASES))
def test_projection_bit_exact_vs_reference_kernel(ab, torch_cuda, case):
    if not oracle.ReferenceGPU.available():
        pytest.skip("reference GPU library not built")
    (g, sh, deg), cam = PROJ_CASES[case]()
    mine = ab.GpuRenderer(g, sh, deg).debug_projection(cam)
    ref = reference_projection(torch_cuda, g, sh, deg, cam)
    np.testing.assert_array_equal(mine["tiles_touched"], ref["tiles_touched"])
    vis = ref["tiles_touched"] > 0
    np.testing.assert_array_equal(mine["rect"][vis], ref["rect"][vis])
    np.testing.assert_array_equal(mine["depth"][vis].view(np.uint32), ref["depth"][vis].view(np.uint32))
    np.testing.assert_array_equal(mine["uv"][vis].view(np.uint32), ref["uv"][vis].view(np.uint32))
    np.testing.assert_array_equal(mine["conic_opacity"][vis].view(np.uint32),
                                  ref["conic_opacity"][vis].view(np.uint32))
    np.testing.assert_array_equal(mine["rgb"][vis].view(np.uint32), ref["rgb"][vis].view(np.uint32))


@pytest.mark.parametrize("case", sorted(PROJ_CASES))
def test_sort_bit_exact_given_same_projection(ab, torch_cuda, case):
    (g, sh, deg), cam = PROJ_CASES[case]()
    r = ab.GpuRenderer(g, sh, deg)
    proj = r.debug_projection(cam)
    tx, ty = (cam.width + 15) // 16, (cam.height + 15) // 16
    tiles, values, ranges = r.debug_sorted(cam, capacity=int(proj["tiles_touched"].astype(np.int64).sum()) + 1024)
    keys = ab.keys_of(tiles, values, proj["depth"])
    # the C restatement of the reference's integer work
    okeys, ovalues, oranges = oracle.Restatement().sort_keys(proj["tiles_touched"], proj["rect"], proj["depth"], tx, ty)
    np.testing.assert_array_equal(keys, okeys)
    np.testing.assert_array_equal(values, ovalues)
    np.testing.assert_array_equal(ranges, oranges)
    # the product's sort alone on that projection
    t2, v2, r2 = ab.sort_projection(proj["tiles_touched"], proj["rect"], proj["depth"], tx, ty)
    np.testing.assert_array_equal(t2, tiles)
    np.testing.assert_array_equal(v2, values)
    np.testing.assert_array_equal(r2, ranges)
    # the reference's own scan + duplicate + CUB sort + tileRanges on that projection
    if oracle.ReferenceGPU.available():
        rkeys, rvalues, rranges = reference_sort(torch_cuda, proj, tx, ty)
        np.testing.assert_array_equal(keys, rkeys)
        np.testing.assert_array_equal(values, rvalues)
        np.testing.assert_array_equal(ranges, rranges)


# ---- working-size scenes -----------------------------------------------------------------------

@pytest.mark.slow
def test_config1_vs_cpu(ab):
    raw = scenes.config(1)[0][0]
    cam = scenes.config(1)[1][0][0]
    g, sh = oracle.Restatement().activate(raw)
    st = {}
    img = ab.GpuRenderer(g, sh, 3).render(cam, st)
    cpu, cst = cpu_render(g, sh, 3, cam)
    assert st["visible"] == cst["visible"] == 60601
    assert_image_parity(img, cpu, "config 1")


@pytest.mark.slow
def test_config2_views_vs_cpu(ab):
    """All 16 ring views of the bench workload against the CPU renderer."""
    (g, sh, deg), cams = config2_scene()
    r = ab.GpuRenderer(g, sh, deg)
    if oracle.ReferenceCPU.available():
        cpu_scene = oracle.ReferenceCPU().scene(g, sh, deg)
        cpu = lambda cam: cpu_scene.render(cam)[0]
    else:
        cpu = lambda cam: cpu_render(g, sh, deg, cam)[0]
    worst = (0, 1e9)
    for cam in cams:
        m, p = assert_image_parity(r.render(cam), cpu(cam), cam.name)
        worst = (max(worst[0], m), min(worst[1], p))
    print("16 ring views: worst max-abs %d/255, worst PSNR %.1f dB" % worst)


def test_pair_overflow_regrows(ab):
    """A frame with more pairs than the initial capacity (2^20) is rendered again after growing."""
    rng = np.random.default_rng(5)
    n = 400
    g = np.zeros((n, 11), np.float32)
    g[:, 0:2] = rng.uniform(-0.5, 0.5, (n, 2))
    g[:, 2] = rng.uniform(3, 4, n)
    g[:, 3:6] = 1.5  # huge: each covers the whole 1920x1080 frame (8160 tiles)
    g[:, 6] = 1
    g[:, 10] = 0.02
    sh = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    cam = scenes.Camera(1920, 1080, 1000.0, 1000.0, 960.0, 540.0, np.eye(3), np.zeros(3))
    st = {}
    img = ab.GpuRenderer(g, sh, 0).render(cam, st)
    assert st["tile_pairs"] > (1 << 20)
    assert_image_parity(img, cpu_render(g, sh, 0, cam)[0], "overflow")


def test_render_device_stream_ordered(ab, torch_cuda):
    torch = torch_cuda
    g, sh, deg = kat.random_cloud(20000)
    r = ab.GpuRenderer(g, sh, deg)
    cams = [kat.gpu_test_camera(320, 240), kat.gpu_test_camera(333, 217)]
    host = [r.render(c) for c in cams]
    stream = torch.cuda.Stream()
    outs = [torch.empty(c.height, c.width, 3, dtype=torch.uint8, device="cuda") for c in cams]
    for c, o in zip(cams, outs):
        r.render_device(c, o.data_ptr(), stream.cuda_stream)
    r.sync()
    for h, o in zip(host, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), h)


@pytest.mark.slow
def test_faster_than_the_reference_gpu_renderer(ab):
    """The same 4 ring views of the 740k-Gaussian scene through the reference's GpuRenderer (its
    own gpu_render.cu, CUB, built for sm_100a as shipped, with --use_fast_math) and through this
    library's drop-in call, both host-to-host (each returns a host image): this one must be faster."""
    import time

    if not oracle.ReferenceGPU.available(fast_math=True):
        pytest.skip("reference GPU library not built")
    raws, camsets = scenes.config(2)
    g, sh = scenes.activate(raws[0])
    cams = camsets[0][:4]
    ref = oracle.ReferenceGPU(fast_math=True)
    h = ref.renderer(g, sh, 3)
    r = ab.GpuRenderer(g, sh, 3)
    try:
        for c in cams:  # warm-up: both grow their buffers
            ref.render(h, c)
            r.render(c)
        t = time.perf_counter()
        for _ in range(3):
            for c in cams:
                ref.render(h, c)
        t_ref = (time.perf_counter() - t) / (3 * len(cams))
        t = time.perf_counter()
        for _ in range(3):
            for c in cams:
                r.render(c)
        t_ours = (time.perf_counter() - t) / (3 * len(cams))
    finally:
        ref.destroy(h)
    print("host-to-host ms/frame: reference GpuRenderer %.3f, aniso_b200 %.3f (%.2fx)"
          % (1e3 * t_ref, 1e3 * t_ours, t_ref / t_ours))
    assert t_ours < t_ref


@pytest.mark.parametrize("w,h", [(1, 1), (7, 5), (17, 9), (3840, 2160)])
def test_image_sizes_vs_cpu(ab, w, h):
    """Frames smaller than one tile, ragged tile edges, and 4K (240 x 135 tiles of 16)."""
    g, sh, deg = kat.random_cloud(20000, seed=9)
    cam = kat.gpu_test_camera(w, h)
    img = ab.GpuRenderer(g, sh, deg).render(cam)
    assert img.shape == (h, w, 3)
    assert_image_parity(img, cpu_render(g, sh, deg, cam)[0], "%dx%d" % (w, h))


def test_empty_scene_renders_black(ab):
    r = ab.GpuRenderer(np.zeros((0, 11), np.float32), np.zeros((0, 48), np.float32), 3)
    st = {}
    img = r.render(kat.gpu_test_camera(320, 240), st)
    assert not img.any() and st["tile_pairs"] == 0 and st["visible"] == 0


def test_degree4_scene_vs_cpu(ab):
    """The loader accepts degree 4 (ply_loader.cpp:67-73); colour is evaluated up to degree 3."""
    g, sh3, _ = kat.random_cloud(8000, seed=10)
    rng = np.random.default_rng(11)
    sh = np.zeros((8000, 25, 3), np.float32)
    sh[:, :16] = sh3.reshape(8000, 16, 3)
    sh[:, 16:] = rng.normal(0, 0.3, (8000, 9, 3))
    cam = kat.gpu_test_camera(256, 192)
    img = ab.GpuRenderer(g, sh.reshape(8000, 75), 4).render(cam)
    assert_image_parity(img, cpu_render(g, sh.reshape(8000, 75), 4, cam)[0], "degree 4")


def test_unchained_launches_render_the_same_bytes(ab, tmp_path):
    """Frames launched with programmatic stream serialisation (the default) and plainly
    (ANISO_B200_CHAIN=0, read once per process, hence a child process) give identical images."""
    import os
    import subprocess
    import sys

    g, sh, d = kat.random_cloud(30000, seed=13)
    cam = kat.gpu_test_camera(640, 360)
    chained = ab.GpuRenderer(g, sh, d).render(cam)
    np.save(tmp_path / "g.npy", g)
    np.save(tmp_path / "sh.npy", sh)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r); import kat, aniso_b200; "
            "g = np.load(%r); sh = np.load(%r); "
            "img = aniso_b200.GpuRenderer(g, sh, %d).render(kat.gpu_test_camera(640, 360)); np.save(%r, img)"
            % (root, os.path.join(root, "tests"), str(tmp_path / "g.npy"), str(tmp_path / "sh.npy"), d,
               str(tmp_path / "img.npy")))
    env = dict(os.environ, ANISO_B200_CHAIN="0")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    np.testing.assert_array_equal(np.load(tmp_path / "img.npy"), chained)
    assert chained.any()


def test_large_host_render_equals_device_render(ab, torch_cuda):
    """Large frames (odd tile-row counts, a ragged last row) rendered into host memory through the
    GpuRenderer::render path equal the same frame rendered into device memory, frame after frame."""
    torch = torch_cuda
    g, sh, deg = kat.random_cloud(60000, seed=14)
    r = ab.GpuRenderer(g, sh, deg)
    for w, h in ((1280, 720), (1000, 1000), (1920, 1080)):
        cam = kat.gpu_test_camera(w, h)
        first = r.render(cam)  # also grows the pair capacity for the device render below
        out = torch.empty(h, w, 3, dtype=torch.uint8, device="cuda")
        r.render_device(cam, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        r.sync()
        dev = out.cpu().numpy()
        np.testing.assert_array_equal(first, dev, err_msg="%dx%d" % (w, h))
        np.testing.assert_array_equal(r.render(cam), dev, err_msg="%dx%d, again" % (w, h))
        assert dev.any()


@pytest.mark.gpu
def test_pinned_host_render_equals_pageable_render(ab, torch_cuda):
    """Pinned host buffers are written by the blend itself (16-byte, 4-byte or single-byte row
    stores, by the alignment of the image rows and the buffer): every byte equals the render into
    pageable memory (a copy of the finished image) and into device memory, and none is left over
    from before."""
    torch = torch_cuda
    g, sh, deg = kat.random_cloud(60000, seed=15)
    r = ab.GpuRenderer(g, sh, deg)
    # 1280: rows of 3840 bytes (16-byte stores); 1284: 3852 (4-byte); 1297: odd (bytes).
    for w, h in ((1280, 720), (1284, 720), (1297, 731), (64, 48)):
        cam = kat.gpu_test_camera(w, h)
        pageable = r.render(cam)
        out = torch.empty(h, w, 3, dtype=torch.uint8, device="cuda")
        r.render_device(cam, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        r.sync()
        np.testing.assert_array_equal(pageable, out.cpu().numpy(), err_msg="%dx%d device" % (w, h))
        n = w * h * 3
        keep = torch.full((n + 16,), 0xAB, dtype=torch.uint8).pin_memory()
        assert keep.is_pinned()
        pinned = keep.numpy()
        for off in (0, 1, 4):  # buffer starts 16-, 1- and 4-byte aligned
            view = pinned[off:off + n].reshape(h, w, 3)
            view[...] = 0xAB
            got = r.render(cam, out=view)
            assert got is view
            np.testing.assert_array_equal(view, pageable, err_msg="%dx%d pinned +%d" % (w, h, off))
        assert pageable.any()


def test_two_scenes_on_two_streams(ab, torch_cuda):
    """Two scenes rendering on two streams at the same time each give their own single renders, and
    one scene whose frames move between streams keeps them in order (they share its buffers)."""
    torch = torch_cuda
    ga, sha, da = kat.random_cloud(30000, seed=21)
    gb, shb, db = kat.random_cloud(20000, seed=22)
    ra, rb = ab.GpuRenderer(ga, sha, da), ab.GpuRenderer(gb, shb, db)
    cams = [kat.gpu_test_camera(320, 240), kat.gpu_test_camera(333, 217), kat.gpu_test_camera(640, 360)]
    want_a = [ra.render(c) for c in cams]
    want_b = [rb.render(c) for c in cams]
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    outs_a = [torch.empty(c.height, c.width, 3, dtype=torch.uint8, device="cuda") for c in cams]
    outs_b = [torch.empty(c.height, c.width, 3, dtype=torch.uint8, device="cuda") for c in cams]
    for _ in range(2):
        for c, oa, ob in zip(cams, outs_a, outs_b):
            ra.render_device(c, oa.data_ptr(), sa.cuda_stream)
            rb.render_device(c, ob.data_ptr(), sb.cuda_stream)
        rb.sync()
        ra.sync()
        for w, o in zip(want_a, outs_a):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
        for w, o in zip(want_b, outs_b):
            np.testing.assert_array_equal(o.cpu().numpy(), w)
    # one scene, its frames alternating between the two streams
    for o in outs_a:
        o.zero_()
    torch.cuda.synchronize()
    for k, (c, o) in enumerate(zip(cams, outs_a)):
        ra.render_device(c, o.data_ptr(), (sa if k % 2 == 0 else sb).cuda_stream)
    ra.sync()
    for w, o in zip(want_a, outs_a):
        np.testing.assert_array_equal(o.cpu().numpy(), w)
