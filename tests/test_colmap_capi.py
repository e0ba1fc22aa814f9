"""aniso_b200_colmap_load (host code of the C ABI, no device needed): COLMAP sparse models in the
binary form the reference reads (camera.cpp:61-140) and in the text form the workload descriptions
are written in, through the same entry point the drop-in CLI's camera loader uses."""
import os
import struct

import numpy as np
import pytest

import aniso_b200
from aniso_b200 import scenes
from aniso_b200._lib import AnisoError


def cams9():
    return scenes.fibonacci_cameras(9, 10.0, scenes.RESOLUTIONS_4, seed=3)


def test_binary_equals_reference_loader(tmp_path, reference_cpu):
    d = str(tmp_path / "sparse")
    scenes.write_colmap(d, cams9(), binary=True, text=False)
    ours = aniso_b200.colmap_load(d)
    ref = reference_cpu.load_colmap(d)  # rows: w h fx fy cx cy R(9) t(3), sorted by image name
    assert len(ours) == len(ref) == 9
    for a, row in zip(ours, ref):
        assert (a.width, a.height) == (row[0], row[1])
        assert (a.fx, a.fy, a.cx, a.cy) == tuple(row[2:6])
        np.testing.assert_array_equal(a.R, row[6:15].reshape(3, 3))  # the same double arithmetic
        np.testing.assert_array_equal(a.t, row[15:18])


def test_text_equals_binary(tmp_path):
    cams = cams9()
    b, t = str(tmp_path / "bin"), str(tmp_path / "txt")
    scenes.write_colmap(b, cams, binary=True, text=False)
    scenes.write_colmap(t, cams, binary=False, text=True)  # %.17g: every double round-trips exactly
    from_bin, from_txt = aniso_b200.colmap_load(b), aniso_b200.colmap_load(t)
    assert [c.name for c in from_txt] == [c.name for c in from_bin] == sorted(c.name for c in cams)
    for x, y in zip(from_txt, from_bin):
        assert (x.width, x.height, x.fx, x.fy, x.cx, x.cy) == (y.width, y.height, y.fx, y.fy, y.cx, y.cy)
        np.testing.assert_array_equal(x.R, y.R)
        np.testing.assert_array_equal(x.t, y.t)
    for x, y in zip(from_txt, scenes.read_colmap_text(t)):  # and the numpy reader
        np.testing.assert_allclose(x.R, y.R, rtol=0, atol=1e-15)


def test_both_present_reads_binary_and_config_workloads(tmp_path):
    d = str(tmp_path / "s")
    cams = scenes.ring_cameras(16, 8.0, 1280, 720, 1100.0)
    scenes.write_colmap(d, cams)
    got = aniso_b200.colmap_load(d)
    assert len(got) == 16 and got[0].name == "ring_000"
    np.testing.assert_allclose(got[0].R, np.eye(3), atol=1e-12)


def test_simple_pinhole_text_and_comments(tmp_path):
    d = tmp_path / "sp"
    d.mkdir()
    (d / "cameras.txt").write_text("# a comment\n\n7 SIMPLE_PINHOLE 640 360 500 320 180\r\n")
    (d / "images.txt").write_text("# images\n3 1 0 0 0 0.5 -1 2 7 b.png\n1.0 2.0 -1\n"
                                  "1 0 0 0 2 0 0 8 7 a.png\n\n")
    got = aniso_b200.colmap_load(str(d))
    assert [c.name for c in got] == ["a.png", "b.png"]
    a, b = got
    assert (a.width, a.height, a.fx, a.fy, a.cx, a.cy) == (640, 360, 500.0, 500.0, 320.0, 180.0)
    np.testing.assert_allclose(b.R, np.eye(3))
    np.testing.assert_array_equal(b.t, [0.5, -1, 2])
    np.testing.assert_allclose(a.R, np.diag([-1.0, -1.0, 1.0]), atol=1e-15)  # (0,0,0,2): 180 degrees about z


def test_errors_follow_the_reference(tmp_path):
    with pytest.raises(AnisoError, match="cameras.txt: cannot open"):
        aniso_b200.colmap_load(str(tmp_path / "missing"))
    d = tmp_path / "dist"
    d.mkdir()
    (d / "cameras.txt").write_text("1 OPENCV 640 480 500 500 320 240 0.1 0.01 0 0\n")
    (d / "images.txt").write_text("1 1 0 0 0 0 0 0 1 x.png\n\n")
    with pytest.raises(AnisoError, match="has lens distortion; undistort the images first"):
        aniso_b200.colmap_load(str(d))
    m = tmp_path / "miss"
    m.mkdir()
    (m / "cameras.txt").write_text("1 PINHOLE 640 480 500 500 320 240\n")
    (m / "images.txt").write_text("1 1 0 0 0 0 0 0 2 x.png\n\n")
    with pytest.raises(AnisoError, match="image x.png refers to a missing camera"):
        aniso_b200.colmap_load(str(m))
    # binary: a truncated cameras.bin, and an unknown model id
    b = tmp_path / "trunc"
    scenes.write_colmap(str(b), cams9(), binary=True, text=False)
    data = (b / "cameras.bin").read_bytes()
    (b / "cameras.bin").write_bytes(data[:-5])
    with pytest.raises(AnisoError, match="cameras.bin: unexpected end of file"):
        aniso_b200.colmap_load(str(b))
    (b / "cameras.bin").write_bytes(struct.pack("<QIiQQ", 1, 1, 42, 64, 48))
    with pytest.raises(AnisoError, match="unknown camera model 42"):
        aniso_b200.colmap_load(str(b))


def test_count_then_fill_and_small_capacity(tmp_path):
    import ctypes

    from aniso_b200 import _lib

    d = str(tmp_path / "s")
    scenes.write_colmap(d, cams9())
    n = ctypes.c_int32(-1)
    assert _lib.lib.aniso_b200_colmap_load(os.fsencode(d), None, 0, ctypes.byref(n)) == _lib.OK and n.value == 9
    arr = (_lib.ColmapCamera * 4)()
    assert _lib.lib.aniso_b200_colmap_load(os.fsencode(d), arr, 4, ctypes.byref(n)) == _lib.ERR_ARGUMENT
    assert "capacity" in _lib.last_error()


def test_dropin_cli_lists_text_and_binary_cameras_alike(tmp_path):
    """The reference CLI, compiled unchanged against the drop-in (`aniso cameras`, main.cpp:105-113),
    reads the text model through the library's loader and prints what it prints for the binary one."""
    import subprocess

    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "aniso_b200_cli")
    if not os.path.exists(cli):
        pytest.skip("drop-in executables not built (no reference sources where the tree was built)")
    cams = cams9()
    t, b = str(tmp_path / "t"), str(tmp_path / "b")
    scenes.write_colmap(t, cams, binary=False, text=True)
    scenes.write_colmap(b, cams, binary=True, text=False)
    out = [subprocess.run([cli, "cameras", d], capture_output=True, text=True, timeout=60) for d in (t, b)]
    assert out[0].returncode == 0 and out[1].returncode == 0, out[0].stderr + out[1].stderr
    assert out[0].stdout.replace(t, "D") == out[1].stdout.replace(b, "D")
    assert "9 cameras" in out[0].stdout
