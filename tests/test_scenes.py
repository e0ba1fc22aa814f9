"""Seeded workload generators and the file formats around the path (3DGS PLY, COLMAP)."""
import os
import tempfile

import numpy as np
import pytest

from aniso_b200 import scenes


def test_generator_is_deterministic_and_has_the_named_distributions():
    a = scenes.make_raw_scene(50_000, (-4, -4, 2), (4, 4, 12), seed=0)
    b = scenes.make_raw_scene(50_000, (-4, -4, 2), (4, 4, 12), seed=0)
    for f in ("xyz", "f_dc", "f_rest", "opacity", "scale", "rot"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert a.xyz[:, 0].min() >= -4 and a.xyz[:, 0].max() <= 4 and a.xyz[:, 2].min() >= 2
    assert abs(a.scale.mean() + 4.0) < 0.01 and abs(a.scale.std() - 0.5) < 0.01
    assert abs(a.opacity.std() - 1.5) < 0.02 and abs(a.f_dc.std() - 0.5) < 0.01
    assert abs(a.f_rest.std() - 0.05) < 0.001 and a.f_rest.shape[1] == 45
    np.testing.assert_allclose(np.linalg.norm(a.rot, axis=1), 1.0, rtol=1e-6)
    assert a.sh_degree == 3


def test_sh_reorder_channel_major_to_coefficient_major():
    raw = scenes.make_raw_scene(3, (0, 0, 0), (1, 1, 1), seed=1)
    k = raw.sh_coeffs()
    # f_rest_0 is coefficient 1 of red, f_rest_15 coefficient 1 of green (ply_loader.cpp:132-138)
    assert k[1, 1, 0] == raw.f_rest[1, 0] and k[1, 1, 1] == raw.f_rest[1, 15] and k[1, 15, 2] == raw.f_rest[1, 44]
    assert np.array_equal(k[:, 0, :], raw.f_dc)


def test_ply_round_trip():
    raw = scenes.make_raw_scene(1000, (-1, -1, -1), (1, 1, 1), seed=3)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.ply")
        scenes.write_ply(p, raw)
        back = scenes.read_ply(p)
    for f in ("xyz", "f_dc", "f_rest", "opacity", "scale", "rot"):
        np.testing.assert_array_equal(getattr(raw, f), getattr(back, f))


def test_colmap_binary_read_by_reference_and_text_round_trip(reference_cpu):
    cams = scenes.fibonacci_cameras(9, 10.0, scenes.RESOLUTIONS_4, seed=3)
    with tempfile.TemporaryDirectory() as d:
        scenes.write_colmap(d, cams)
        got = reference_cpu.load_colmap(d)
        txt = scenes.read_colmap_text(d)
    by_name = sorted(cams, key=lambda c: c.name)
    for row, c, t in zip(got, by_name, txt):
        assert (row[0], row[1]) == (c.width, c.height)
        np.testing.assert_allclose(row[2:6], [c.fx, c.fy, c.cx, c.cy])
        np.testing.assert_allclose(row[6:15].reshape(3, 3), c.R, atol=1e-12)
        np.testing.assert_allclose(row[15:18], c.t, atol=1e-12)
        np.testing.assert_allclose(t.R, c.R, atol=1e-12)
        np.testing.assert_allclose(t.t, c.t, atol=1e-12)
        assert (t.width, t.height, t.fx) == (c.width, c.height, c.fx)


def test_ring_camera_zero_is_identity_pose():
    c = scenes.ring_cameras(16, 8.0, 1280, 720, 1100.0)[0]
    np.testing.assert_allclose(c.R, np.eye(3), atol=1e-12)
    np.testing.assert_allclose(c.t, [0, 0, 8], atol=1e-12)
    np.testing.assert_allclose(c.centre(), [0, 0, -8], atol=1e-12)


@pytest.mark.parametrize("k,views", [(1, [1]), (2, [16]), (3, [1]), (4, [64]), (5, [4] * 8)])
def test_workload_shapes(k, views):
    scs, cams = scenes.config(k, scale=0.001)
    assert [len(v) for v in cams] == views
    if k == 4:
        assert {(c.width, c.height) for c in cams[0]} <= set(scenes.RESOLUTIONS_4)
        assert all(abs(c.fx - 0.9 * c.width) < 1e-9 for c in cams[0])


def test_colmap_binary_reader_equals_reference_loader(tmp_path, reference_cpu):
    cams = scenes.fibonacci_cameras(9, 10.0, scenes.RESOLUTIONS_4, seed=3)
    d = str(tmp_path / "sparse")
    scenes.write_colmap(d, cams)
    ours = scenes.read_colmap_binary(d)
    ref = reference_cpu.load_colmap(d)
    assert len(ours) == len(ref) == 9
    assert [c.name for c in ours] == sorted(c.name for c in cams)
    for a, row in zip(ours, ref):  # rows: width height fx fy cx cy R(9) t(3), sorted by image name
        assert (a.width, a.height) == (row[0], row[1])
        assert (a.fx, a.fy, a.cx, a.cy) == tuple(row[2:6])
        np.testing.assert_array_equal(np.asarray(a.R), row[6:15].reshape(3, 3))  # same double arithmetic
        np.testing.assert_array_equal(np.asarray(a.t), row[15:18])


def test_read_colmap_picks_either_form(tmp_path):
    cams = scenes.ring_cameras(5, 8.0, 640, 360, 500.0)
    for binary, text in ((True, False), (False, True)):
        d = str(tmp_path / ("b" if binary else "t"))
        scenes.write_colmap(d, cams, binary=binary, text=text)
        got = scenes.read_colmap(d)
        assert [c.name for c in got] == sorted(c.name for c in cams)
        for a in got:
            b = next(c for c in cams if c.name == a.name)
            np.testing.assert_allclose(np.asarray(a.R), np.asarray(b.R), atol=1e-12)
            np.testing.assert_allclose(np.asarray(a.t), np.asarray(b.t), atol=1e-12)
