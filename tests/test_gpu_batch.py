"""Batches (many views of several scenes in one launch sequence) against single-view renders.

A batch view must be bit-identical to the same view rendered alone: every stage computes the same
per-entry values, and the sort orders each tile's pairs by (depth bits, Gaussian index) as the
single-view sort does. The image does not depend on the tile shape (8x8, 16x16, 16x32) or the
blend batch, because each pixel's splat list is the CPU renderer's 8x8-tile list whatever the
shape. The training batch adds each view's gradient to its scene in view order, so it equals the
single-view gradients summed in the same order, bit for bit.
"""
import numpy as np
import pytest

import kat
from aniso_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ab():
    import aniso_b200

    assert aniso_b200.GpuRenderer.available(), "no CUDA device"
    return aniso_b200


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def mixed_views():
    """Three scenes of uneven size (one empty) and seven views of uneven resolution."""
    clouds = [kat.random_cloud(20000, seed=1), kat.random_cloud(7000, seed=2),
              (np.zeros((0, 11), np.float32), np.zeros((0, 48), np.float32), 3)]
    sizes = [(320, 240), (333, 217), (160, 96), (257, 129), (320, 240), (64, 48), (200, 150)]
    view_scene = [0, 0, 0, 1, 1, 2, 2]
    cams = []
    for k, (w, h) in enumerate(sizes):
        c = kat.gpu_test_camera(w, h)
        yaw = 0.05 * (k - 3)
        R = np.array([[np.cos(yaw), 0, np.sin(yaw)], [0, 1, 0], [-np.sin(yaw), 0, np.cos(yaw)]])
        cams.append(scenes.Camera(w, h, c.fx, c.fy, c.cx, c.cy, R @ np.asarray(c.R), np.asarray(c.t)))
    return clouds, view_scene, cams


def render_batch(ab, torch, renderers, view_scene, cams, options, stream=None):
    """Renders the batch; a first frame whose pairs exceeded the starting capacity is rendered
    again (the batch API's contract: the capacity has been grown by then)."""
    b = ab.BatchRenderer(renderers, view_scene, options)
    outs = [torch.full((c.height, c.width, 3), 7, dtype=torch.uint8, device="cuda") for c in cams]
    s = stream or torch.cuda.current_stream()
    for attempt in range(3):
        b.render_device(cams, [o.data_ptr() for o in outs], s.cuda_stream)
        try:
            st = b.sync()
            break
        except ab.AnisoError as e:
            if "pair capacity exceeded" not in str(e) or attempt == 2:
                raise
    return b, [o.cpu().numpy() for o in outs], st


def test_batch_views_equal_single_renders(ab, torch):
    clouds, view_scene, cams = mixed_views()
    rs = [ab.GpuRenderer(g, sh, d) for g, sh, d in clouds]
    single = [rs[s].render(c) for s, c in zip(view_scene, cams)]
    _, imgs, st = render_batch(ab, torch, rs, view_scene, cams, ab.BatchOptions())
    for k, (a, b) in enumerate(zip(imgs, single)):
        np.testing.assert_array_equal(a, b, err_msg="view %d" % k)
    assert not imgs[5].any() and not imgs[6].any()  # the empty scene renders black
    assert st["tile_pairs"] > 0


def test_scenes_of_different_degrees_in_one_batch(ab, torch):
    """Each view is coloured at its own scene's degree, as a single render of that scene is."""
    g3, sh3, _ = kat.random_cloud(6000, seed=7)
    g1, sh1 = g3[:4000].copy(), np.ascontiguousarray(sh3[:4000].reshape(4000, 16, 3)[:, :4]).reshape(4000, 12)
    g0, sh0 = g3[2000:].copy(), np.ascontiguousarray(sh3[2000:].reshape(4000, 16, 3)[:, :1]).reshape(4000, 3)
    rs = [ab.GpuRenderer(g3, sh3, 3), ab.GpuRenderer(g1, sh1, 1), ab.GpuRenderer(g0, sh0, 0)]
    cams = [kat.gpu_test_camera(160, 120), kat.gpu_test_camera(200, 150), kat.gpu_test_camera(128, 96)]
    view_scene = [0, 1, 2]
    for opt in (3, 2):
        single = [rs[s].render(c, options=ab.RenderOptions(sh_degree=opt)) for s, c in zip(view_scene, cams)]
        _, imgs, _ = render_batch(ab, torch, rs, view_scene, cams, ab.BatchOptions(sh_degree=opt))
        for k, (a, b) in enumerate(zip(imgs, single)):
            np.testing.assert_array_equal(a, b, err_msg="view %d, option %d" % (k, opt))


def test_more_views_than_staged_cameras(ab, torch):
    """A scene seen by more views than the preprocess kernel keeps in shared memory (64)."""
    g, sh, d = kat.random_cloud(3000, seed=8)
    r = ab.GpuRenderer(g, sh, d)
    cams = [kat.gpu_test_camera(64 + (k % 5) * 8, 48 + (k % 3) * 8) for k in range(80)]
    _, imgs, _ = render_batch(ab, torch, [r], [0] * 80, cams, ab.BatchOptions(use_graph=True))
    for k in (0, 63, 64, 79):
        np.testing.assert_array_equal(imgs[k], r.render(cams[k]), err_msg="view %d" % k)


@pytest.mark.parametrize("tile,batch,bits", [((8, 8), 128, 8), ((8, 8), 256, 9), ((16, 16), 128, 9),
                                             ((16, 16), 256, 9), ((16, 32), 256, 8), ((16, 32), 512, 9)])
def test_image_independent_of_launch_shape(ab, torch, tile, batch, bits):
    clouds, view_scene, cams = mixed_views()
    rs = [ab.GpuRenderer(g, sh, d) for g, sh, d in clouds]
    single = [rs[s].render(c) for s, c in zip(view_scene, cams)]
    _, imgs, _ = render_batch(ab, torch, rs, view_scene, cams,
                              ab.BatchOptions(tile=tile, blend_batch=batch, radix_bits=bits))
    for k, (a, b) in enumerate(zip(imgs, single)):
        np.testing.assert_array_equal(a, b, err_msg="view %d, tile %s, %d-bit digits" % (k, tile, bits))


@pytest.mark.parametrize("tile", [(16, 16), (8, 8)])
def test_many_tiles_with_nine_bit_digits(ab, torch, tile):
    """72,000 tiles of 16x16 (17 key bits: tile passes of 9 + 8 bits) or 288,000 of 8x8 (19 bits:
    9 + 9 + 8): the batch sorts with the fewest passes 9-bit digits allow, images as single renders."""
    g, sh, d = kat.random_cloud(20000, seed=11)
    r = ab.GpuRenderer(g, sh, d)
    cams = []
    for k in range(20):
        c = kat.gpu_test_camera(1280, 720)
        yaw = 0.02 * (k - 10)
        R = np.array([[np.cos(yaw), 0, np.sin(yaw)], [0, 1, 0], [-np.sin(yaw), 0, np.cos(yaw)]])
        cams.append(scenes.Camera(1280, 720, c.fx, c.fy, c.cx, c.cy, R @ np.asarray(c.R), np.asarray(c.t)))
    _, nine, _ = render_batch(ab, torch, [r], [0] * 20, cams, ab.BatchOptions(tile=tile, radix_bits=9))
    _, eight, _ = render_batch(ab, torch, [r], [0] * 20, cams, ab.BatchOptions(tile=tile, radix_bits=8))
    for k in range(20):
        np.testing.assert_array_equal(nine[k], eight[k], err_msg="view %d" % k)
    for k in (0, 7, 19):
        np.testing.assert_array_equal(nine[k], r.render(cams[k]), err_msg="view %d" % k)
    assert any(img.any() for img in nine)


def test_batch_of_near_and_far_scenes(ab, torch):
    """A scene with Gaussians past depth 8192 makes the whole batch sort depths with four 8-bit
    passes; its views still equal single renders, which for the near scene take three 9-bit ones."""
    near = kat.random_cloud(8000, seed=21)
    g, sh, d = kat.random_cloud(8000, seed=22)
    g = g.copy()
    ratio = np.float32(12000.0) / g[:500, 2]
    g[:500, 0] *= ratio
    g[:500, 1] *= ratio
    g[:500, 2] = 12000.0  # on screen and visible, past 8192
    rs = [ab.GpuRenderer(*near), ab.GpuRenderer(g, sh, d)]
    cams = [kat.gpu_test_camera(320, 240), kat.gpu_test_camera(333, 217), kat.gpu_test_camera(320, 240)]
    view_scene = [0, 1, 1]
    single = [rs[s].render(c) for s, c in zip(view_scene, cams)]
    for graph in (False, True):
        _, imgs, _ = render_batch(ab, torch, rs, view_scene, cams, ab.BatchOptions(use_graph=graph))
        for k, (a, b) in enumerate(zip(imgs, single)):
            np.testing.assert_array_equal(a, b, err_msg="view %d, graph %s" % (k, graph))


def test_graph_batch_follows_cameras_across_the_depth_limit(ab, torch):
    """A recorded batch whose cameras move back past depth 8192 (and forward again) is recorded
    again for the other depth passes; every replay equals the single renders."""
    g, sh, d = kat.random_cloud(6000, seed=23)
    r = ab.GpuRenderer(g, sh, d)
    b = ab.BatchRenderer([r], [0, 0], ab.BatchOptions(use_graph=True))
    for tz in (0.0, 9000.0, 0.0):
        cams = []
        for w, h in ((320, 240), (256, 160)):
            c = kat.gpu_test_camera(w, h)
            f = c.fx * (1.0 + tz / 5.0)  # a longer lens keeps the cloud's size on screen
            cams.append(scenes.Camera(w, h, f, f, c.cx, c.cy, np.asarray(c.R), np.array([0.0, 0.0, tz])))
        outs = [torch.zeros((c.height, c.width, 3), dtype=torch.uint8, device="cuda") for c in cams]
        for attempt in range(3):
            b.render_device(cams, [o.data_ptr() for o in outs], torch.cuda.current_stream().cuda_stream)
            try:
                b.sync()
                break
            except ab.AnisoError as e:
                if "pair capacity exceeded" not in str(e) or attempt == 2:
                    raise
        for k, c in enumerate(cams):
            single = r.render(c)
            assert single.any()
            np.testing.assert_array_equal(outs[k].cpu().numpy(), single, err_msg="view %d, tz %g" % (k, tz))


def test_frame_kernel_count(ab):
    """A small frame: the frame's start (the tables' upload and frame_begin's clears in one
    kernel), preprocess (which also counts the first depth pass's digits), the multi-kernel sort
    (the default): the first depth pass (span scan + downsweep), two more of upsweep + span
    scan + downsweep (three when a depth can reach 8192: the scene's box decides), pair count /
    offsets / expansion, then for at most 4096 tiles the tile binning (scan + scatter, which also
    write the ranges), else the first tile pass (2 kernels: the expansion counted its digits), any
    second one (3) and the ranges; blend. With ANISO_B200_SORT=persistent the sort is one
    cooperative launch instead (depth passes, pair expansion, tile passes, ranges)."""
    import os

    multi = os.environ.get("ANISO_B200_SORT") != "persistent"
    g, sh, d = kat.random_cloud(5000, seed=3)
    r = ab.GpuRenderer(g, sh, d)
    r.render(kat.gpu_test_camera(320, 240))  # 300 tiles: binned
    assert r.frame_kernels() == (1 + 1 + 2 + 2 * 3 + 3 + 2 + 1 if multi else 4)
    r.render(kat.gpu_test_camera(64, 48))  # 12 tiles: binned
    assert r.frame_kernels() == (1 + 1 + 2 + 2 * 3 + 3 + 2 + 1 if multi else 4)
    r.render(kat.gpu_test_camera(1920, 1088))  # 8160 tiles: two LSD tile passes
    assert r.frame_kernels() == (1 + 1 + 2 + 2 * 3 + 3 + 2 + 3 + 1 + 1 if multi else 4)
    g = g.copy()
    g[0, :3] = (0.0, 0.0, 9000.0)  # one Gaussian (on the axis, visible) past 8192: four depth passes
    far = ab.GpuRenderer(g, sh, d)
    far.render(kat.gpu_test_camera(320, 240))
    assert far.frame_kernels() == (1 + 1 + 2 + 3 * 3 + 3 + 2 + 1 if multi else 4)


def test_large_batch_counts_digits_in_separate_passes(ab, torch):
    """Above 4M entries the sort counts digits with its own kernels instead of in the kernels that
    write the keys (the per-view frames below it use the latter): both give the same images."""
    g, sh, d = kat.random_cloud(300000, seed=12)
    r = ab.GpuRenderer(g, sh, d)
    cams = []
    for k in range(16):
        c = kat.gpu_test_camera(640, 360)
        yaw = 0.03 * (k - 8)
        R = np.array([[np.cos(yaw), 0, np.sin(yaw)], [0, 1, 0], [-np.sin(yaw), 0, np.cos(yaw)]])
        cams.append(scenes.Camera(640, 360, c.fx, c.fy, c.cx, c.cy, R @ np.asarray(c.R), np.asarray(c.t)))
    _, imgs, st = render_batch(ab, torch, [r], [0] * 16, cams, ab.BatchOptions())
    for k in range(16):
        np.testing.assert_array_equal(imgs[k], r.render(cams[k]), err_msg="view %d" % k)
    assert st["tile_pairs"] > 0


def test_graph_replay_follows_new_cameras(ab, torch):
    clouds, view_scene, cams = mixed_views()
    rs = [ab.GpuRenderer(g, sh, d) for g, sh, d in clouds]
    b = ab.BatchRenderer(rs, view_scene, ab.BatchOptions(use_graph=True))
    outs = [torch.empty((c.height, c.width, 3), dtype=torch.uint8, device="cuda") for c in cams]
    ptrs = [o.data_ptr() for o in outs]
    stream = torch.cuda.Stream()
    for shift in (0.0, 0.3, -0.2):  # records once, then replays with new poses
        moved = [scenes.Camera(c.width, c.height, c.fx, c.fy, c.cx, c.cy, np.asarray(c.R),
                               np.asarray(c.t) + np.array([shift, 0.1 * shift, 0.0])) for c in cams]
        b.render_device(moved, ptrs, stream.cuda_stream)
        b.sync()
        for k, (o, s) in enumerate(zip(outs, view_scene)):
            np.testing.assert_array_equal(o.cpu().numpy(), rs[s].render(moved[k]), err_msg="shift %g view %d" % (shift, k))
    # New image sizes record the graph again.
    small = [scenes.Camera(c.width // 2 + 1, c.height // 2 + 1, c.fx / 2, c.fy / 2, c.cx / 2, c.cy / 2,
                           np.asarray(c.R), np.asarray(c.t)) for c in cams]
    outs2 = [torch.empty((c.height, c.width, 3), dtype=torch.uint8, device="cuda") for c in small]
    b.render_device(small, [o.data_ptr() for o in outs2], stream.cuda_stream)
    b.sync()
    for k, (o, s) in enumerate(zip(outs2, view_scene)):
        np.testing.assert_array_equal(o.cpu().numpy(), rs[s].render(small[k]))


def test_batch_overflow_regrows(ab, torch):
    """Two views whose pairs together exceed the batch's first pair capacity."""
    rng = np.random.default_rng(5)
    n = 300
    g = np.zeros((n, 11), np.float32)
    g[:, 0:2] = rng.uniform(-0.5, 0.5, (n, 2))
    g[:, 2] = rng.uniform(3, 4, n)
    g[:, 3:6] = 1.5
    g[:, 6] = 1
    g[:, 10] = 0.02
    sh = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    r = ab.GpuRenderer(g, sh, 0)
    cams = [scenes.Camera(1920, 1080, 1000.0, 1000.0, 960.0, 540.0, np.eye(3), np.zeros(3)),
            scenes.Camera(1280, 720, 700.0, 700.0, 640.0, 360.0, np.eye(3), np.zeros(3))]
    b = ab.BatchRenderer([r], [0, 0])
    outs = [torch.empty((c.height, c.width, 3), dtype=torch.uint8, device="cuda") for c in cams]
    stream = torch.cuda.current_stream().cuda_stream
    b.render_device(cams, [o.data_ptr() for o in outs], stream)
    with pytest.raises(ab.AnisoError, match="pair capacity exceeded"):
        b.sync()
    b.render_device(cams, [o.data_ptr() for o in outs], stream)  # grown: renders now
    st = b.sync()
    assert st["tile_pairs"] > (1 << 20)
    for o, c in zip(outs, cams):
        np.testing.assert_array_equal(o.cpu().numpy(), r.render(c))


def make_params(torch, n, seed):
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(-1, 1, n), rng.uniform(-0.7, 0.7, n), rng.uniform(3, 6, n)], 1)
    arrs = [means, rng.normal(-2.6, 0.4, (n, 3)), rng.normal(0, 1, (n, 4)), rng.normal(0, 1, n),
            rng.normal(0, 0.3, (n, 16, 3))]
    return [torch.tensor(a, dtype=torch.float32, device="cuda", requires_grad=True) for a in arrs]


def test_train_batch_equals_single_views(ab, torch):
    from aniso_b200.autograd import rasterize, rasterize_batch

    params = [make_params(torch, 300, 0), make_params(torch, 150, 1)]
    base = [scenes.Camera(96, 64, 80.0, 80.0, 48.0, 32.0, np.eye(3), np.zeros(3)),
            scenes.Camera(80, 60, 70.0, 70.0, 40.0, 30.0, np.eye(3), np.array([0.1, 0.0, 0.0])),
            scenes.Camera(64, 64, 60.0, 60.0, 32.0, 32.0, np.eye(3), np.array([-0.1, 0.05, 0.0]))]
    view_scene = [0, 0, 1]
    rng = np.random.default_rng(3)
    targets = [torch.tensor(rng.uniform(0, 1, (c.height, c.width, 3)), dtype=torch.float32, device="cuda")
               for c in base]

    imgs = rasterize_batch(params, base, view_scene)
    sum(((i - t) ** 2).sum() for i, t in zip(imgs, targets)).backward()
    batch_img = [i.detach().cpu().numpy() for i in imgs]
    batch_grad = [[p.grad.cpu().numpy() for p in ps] for ps in params]

    for ps in params:
        for p in ps:
            p.grad = None
    single_img = []
    for k, (c, s) in enumerate(zip(base, view_scene)):
        img = rasterize(*params[s], c)
        ((img - targets[k]) ** 2).sum().backward()  # .grad accumulates over views in view order
        single_img.append(img.detach().cpu().numpy())
    for a, b in zip(batch_img, single_img):
        np.testing.assert_array_equal(a, b)
    for gs, ps in zip(batch_grad, params):
        for a, p in zip(gs, ps):
            np.testing.assert_array_equal(a, p.grad.cpu().numpy())
