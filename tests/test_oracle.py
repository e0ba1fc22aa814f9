"""The oracle is pinned before it is trusted: the C restatement must reproduce the reference's
own outputs bit for bit -- against the committed golden fixtures (always) and against the
reference library compiled from its sources (where it was built)."""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

import kat
import oracle
from aniso_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    arrays = np.load(os.path.join(GOLDEN, "reference_cpu.npz"))
    with open(os.path.join(GOLDEN, "reference_cpu.json")) as f:
        meta = json.load(f)
    return arrays, meta


# ---- restatement vs golden fixtures (reference outputs) ----------------------------------------

@pytest.mark.parametrize("name", ["kat_single", "kat_front_back", "kat_behind"])
def test_kat_images_match_golden(restatement, golden, name):
    arrays, meta = golden
    g, sh, deg = getattr(kat, name)()
    img, st = restatement.render(g, sh, deg, kat.kat_camera())
    np.testing.assert_array_equal(img, arrays[name + "_image"])
    assert st["visible"] == meta[name]["visible"] and st["tile_pairs"] == meta[name]["tile_pairs"]


def test_cloud_matches_golden(restatement, golden):
    arrays, meta = golden
    g, sh, deg = kat.random_cloud(1500, seed=21)
    assert sha(g) + sha(sh) == meta["cloud"]["inputs_sha256"], "scene generator drifted"
    cam = kat.gpu_test_camera(160, 120)
    img, st = restatement.render(g, sh, deg, cam)
    np.testing.assert_array_equal(img, arrays["cloud_image"])
    splats, radius, alive = restatement.make_splats(g, sh, deg, cam)
    np.testing.assert_array_equal(alive.astype(np.uint8), arrays["cloud_alive"])
    np.testing.assert_array_equal(radius[alive], arrays["cloud_radius"][alive])
    np.testing.assert_array_equal(splats[alive].view(np.uint32), arrays["cloud_splats"][alive].view(np.uint32))
    for d, s in [(0, 1.0), (1, 0.7), (2, 1.3)]:
        im, _ = restatement.render(g, sh, deg, cam, d, s)
        assert sha(im) == meta["cloud_deg%d_scale%g" % (d, s)]["sha256"]


def test_sh_colors_match_golden(restatement, golden):
    arrays, _ = golden
    for i, d in enumerate(arrays["sh_dirs"]):
        for deg in range(4):
            np.testing.assert_array_equal(restatement.sh_color(arrays["sh_coeffs"], 3, d, deg),
                                          arrays["sh_colors"][i, deg])


def test_activation_matches_golden(restatement, golden):
    arrays, meta = golden
    raw = scenes.make_raw_scene(200, (-1, -1, 2), (1, 1, 4), seed=9)
    assert sha(raw.xyz) + sha(raw.f_rest) + sha(raw.rot) == meta["activation"]["inputs_sha256"]
    g, sh = restatement.activate(raw)
    np.testing.assert_array_equal(g.view(np.uint32), arrays["act_gauss"].view(np.uint32))
    np.testing.assert_array_equal(sh.view(np.uint32), arrays["act_sh"].view(np.uint32))


@pytest.mark.slow
@pytest.mark.parametrize("k", [1, 2])
def test_working_size_view0_matches_golden(restatement, golden, k):
    """Full-size images: size-independent pin through their SHA-256 and counts."""
    arrays, meta = golden
    scs, cams = scenes.config(k)
    g, sh = restatement.activate(scs[0])
    img, st = restatement.render(g, sh, 3, cams[0][0])
    m = meta["config%d_view0" % k]
    assert st["visible"] == m["visible"] and st["tile_pairs"] == m["tile_pairs"]
    assert sha(img) == m["sha256"]
    np.testing.assert_array_equal(img[100:164, 200:264], arrays["config%d_view0_crop" % k])


# ---- the reference's known-answer tests on the restatement (test_render.cpp, test_sh.cpp) ----

def test_kat_analytic_centre_pixel(restatement):
    g, sh, deg = kat.kat_single()
    img, _ = restatement.render(g, sh, deg, kat.kat_camera())
    variance = np.float32(3.2) ** 2 + np.float32(0.3)
    expected = 0.8 * np.exp(-0.5 * 0.5 / variance) * 255.0
    assert abs(int(img[32, 32, 0]) - int(expected + 0.5)) <= 1
    assert img[32, 32, 1] == 0 and img[2, 2, 0] == 0


def test_kat_sh_basis(restatement):
    sh = np.zeros(48, np.float32)
    sh[0] = 0.4
    for d in ([1, 0, 0], [0, 0, -1]):
        c = restatement.sh_color(sh, 3, d, 3)
        assert abs(c[0] - (0.5 + 0.28209479177387814 * 0.4)) < 1e-5 and abs(c[1] - 0.5) < 1e-5
    sh = np.zeros(48, np.float32)
    sh[1 * 3 + 1] = 0.5
    c1 = 0.4886025119029199
    assert abs(restatement.sh_color(sh, 3, [0, -1, 0], 3)[1] - (0.5 + c1 * 0.5)) < 1e-5
    assert abs(restatement.sh_color(sh, 3, [0, 1, 0], 3)[1] - (0.5 - c1 * 0.5)) < 1e-5
    assert abs(restatement.sh_color(sh, 3, [1, 0, 0], 3)[1] - 0.5) < 1e-5
    assert abs(restatement.sh_color(sh, 3, [0, -1, 0], 0)[1] - 0.5) < 1e-5
    sh = np.zeros(48, np.float32)
    sh[2] = -10
    assert restatement.sh_color(sh, 3, [0, 0, 1], 3)[2] == 0.0


# ---- restatement vs the reference library itself (where it was built) ------------------------

CASES = [("cloud", lambda: kat.random_cloud(3000, seed=1), kat.gpu_test_camera(213, 157), 3, 1.0),
         ("cloud_deg1", lambda: kat.random_cloud(3000, seed=2), kat.gpu_test_camera(128, 96), 1, 0.5),
         ("front_back", kat.kat_front_back, kat.kat_camera(), 3, 1.0)]


@pytest.mark.parametrize("name,make,cam,deg_opt,scale", CASES, ids=[c[0] for c in CASES])
def test_restatement_equals_reference_bitwise(restatement, reference_cpu, name, make, cam, deg_opt, scale):
    g, sh, deg = make()
    a, sa = restatement.render(g, sh, deg, cam, deg_opt, scale)
    b, sb = reference_cpu.render(g, sh, deg, cam, deg_opt, scale)
    np.testing.assert_array_equal(a, b)
    assert sa["visible"] == sb["visible"] and sa["tile_pairs"] == sb["tile_pairs"]
    x, rx, ax = restatement.make_splats(g, sh, deg, cam, deg_opt, scale)
    y, ry, ay = reference_cpu.make_splats(g, sh, deg, cam, deg_opt, scale)
    np.testing.assert_array_equal(ax, ay)
    np.testing.assert_array_equal(x[ax].view(np.uint32), y[ay].view(np.uint32))
    np.testing.assert_array_equal(rx[ax], ry[ay])


def test_restatement_activation_equals_reference_loader(restatement, reference_cpu):
    for deg in (0, 1, 3):
        raw = scenes.make_raw_scene(500, (-1, -1, 1), (1, 1, 3), seed=deg, sh_degree=deg)
        with tempfile.TemporaryDirectory() as tmp:
            p = os.path.join(tmp, "s.ply")
            scenes.write_ply(p, raw)
            g2, sh2, d2 = reference_cpu.load_ply(p)
        g, sh = restatement.activate(raw)
        assert d2 == deg
        np.testing.assert_array_equal(g.view(np.uint32), g2.view(np.uint32))
        np.testing.assert_array_equal(sh.view(np.uint32), sh2.view(np.uint32))


def test_camera_centre_equals_reference(restatement, reference_cpu):
    for cam in scenes.ring_cameras(7, 5.0, 64, 48, 50.0):
        np.testing.assert_array_equal(restatement.camera_centre(cam), reference_cpu.camera_centre(cam))


# ---- the restatement of the GPU path's integer work -------------------------------------------

def _projection(n, tiles_x, tiles_y, seed):
    rng = np.random.default_rng(seed)
    x0 = rng.integers(0, tiles_x, n)
    y0 = rng.integers(0, tiles_y, n)
    x1 = np.minimum(tiles_x - 1, x0 + rng.integers(0, 4, n))
    y1 = np.minimum(tiles_y - 1, y0 + rng.integers(0, 3, n))
    rect = np.stack([x0, y0, x1, y1], 1).astype(np.uint32)
    tt = ((x1 - x0 + 1) * (y1 - y0 + 1)).astype(np.uint32)
    tt[rng.random(n) < 0.3] = 0  # culled
    depth = rng.choice(np.float32([0.5, 1.0, 2.0, 3.25]), n) if seed % 2 else rng.uniform(0.2, 40, n)
    return tt, rect, depth.astype(np.float32)


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_sort_keys_restatement_properties(restatement, seed):
    """Sorted by (tile, depth bits, index); ranges delimit each tile's run; empty tiles {0, 0}."""
    tx, ty = 13, 7
    tt, rect, depth = _projection(3000, tx, ty, seed)
    keys, values, ranges = restatement.sort_keys(tt, rect, depth, tx, ty)
    assert len(keys) == int(tt.sum())
    order = np.lexsort((values, keys))  # by key, then index: what a stable sort of index order gives
    np.testing.assert_array_equal(order, np.arange(len(keys)))
    tiles = (keys >> np.uint64(32)).astype(np.int64)
    for t in range(tx * ty):
        idx = np.nonzero(tiles == t)[0]
        if len(idx) == 0:
            assert tuple(ranges[t]) == (0, 0)
        else:
            assert tuple(ranges[t]) == (idx[0], idx[-1] + 1)
    np.testing.assert_array_equal(keys & np.uint64(0xFFFFFFFF), depth.view(np.uint32)[values].astype(np.uint64))
