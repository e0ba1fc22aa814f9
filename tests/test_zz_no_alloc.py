"""aniso_b200_sort_projection_noalloc against aniso_b200_sort_projection (needs a GPU).

The no-alloc variant keeps its work buffers in one static device array, so it is checked on two
calls in a row (the second call must not see anything the first one left behind) and against the
allocating entry point on the same projection, bit for bit. This file is named to be collected
last, so the static array is exercised after every other test has used the device as well.
"""
import ctypes

import numpy as np
import pytest

import kat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import aniso_b200
    from aniso_b200 import _lib

    assert torch.cuda.is_available()
    return torch, aniso_b200, _lib


def projection(ab, n=20000, w=320, h=240, seed=1):
    g, sh, deg = kat.random_cloud(n, seed=seed)
    cam = kat.gpu_test_camera(w, h)
    proj = ab.GpuRenderer(g, sh, deg).debug_projection(cam)
    return proj, (w + 15) // 16, (h + 15) // 16


def call(torch, _lib, proj, tx, ty, capacity, stream):
    dev = lambda a, dt: torch.tensor(np.ascontiguousarray(a).view(dt), device="cuda")
    n = proj["depth"].shape[0]
    tt = dev(proj["tiles_touched"].astype(np.uint32), np.int32)
    rect = dev(proj["rect"].astype(np.uint32).reshape(-1), np.int32)
    depth = dev(proj["depth"].astype(np.float32), np.float32)
    tiles = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device="cuda")
    values = torch.full((max(capacity, 1),), -7, dtype=torch.int32, device="cuda")
    ranges = torch.full((tx * ty * 2,), -7, dtype=torch.int32, device="cuda")
    pairs = torch.zeros(1, dtype=torch.int64, device="cuda")
    P = ctypes.c_void_p
    rc = _lib.lib.aniso_b200_sort_projection_noalloc(
        n, P(tt.data_ptr()), P(rect.data_ptr()), P(depth.data_ptr()), tx, ty, P(tiles.data_ptr()),
        P(values.data_ptr()), capacity, P(ranges.data_ptr()), P(pairs.data_ptr()), P(stream.cuda_stream))
    assert rc == _lib.OK, _lib.last_error()
    stream.synchronize()
    u32 = lambda t: t.cpu().numpy().view(np.uint32)
    return u32(tiles), u32(values), u32(ranges).reshape(-1, 2), int(pairs.cpu().numpy().view(np.uint64)[0])


def test_matches_allocating_sort_twice_in_a_row(env):
    torch, ab, _lib = env
    proj, tx, ty = projection(ab)
    ref_tiles, ref_values, ref_ranges = ab.sort_projection(proj["tiles_touched"], proj["rect"], proj["depth"], tx, ty)
    P = len(ref_values)
    assert P > 0
    stream = torch.cuda.Stream()
    for _ in range(2):
        tiles, values, ranges, pairs = call(torch, _lib, proj, tx, ty, P + 64, stream)
        assert pairs == P
        np.testing.assert_array_equal(tiles[:P], ref_tiles)
        np.testing.assert_array_equal(values[:P], ref_values)
        np.testing.assert_array_equal(ranges, ref_ranges)
        assert (tiles[P:] == np.uint32(0xFFFFFFF9)).all()  # nothing written past the pairs


def test_second_projection_after_first(env):
    """A smaller second problem right after a larger one sees none of the first one's state."""
    torch, ab, _lib = env
    stream = torch.cuda.Stream()
    big, tx, ty = projection(ab, 30000, 333, 217, seed=4)
    call(torch, _lib, big, tx, ty, 1 << 20, stream)
    small, tx2, ty2 = projection(ab, 3000, 200, 150, seed=5)
    ref = ab.sort_projection(small["tiles_touched"], small["rect"], small["depth"], tx2, ty2)
    tiles, values, ranges, pairs = call(torch, _lib, small, tx2, ty2, len(ref[1]) + 8, stream)
    assert pairs == len(ref[1])
    np.testing.assert_array_equal(tiles[:pairs], ref[0])
    np.testing.assert_array_equal(values[:pairs], ref[1])
    np.testing.assert_array_equal(ranges, ref[2])


def test_pairs_beyond_capacity_are_not_written(env):
    torch, ab, _lib = env
    proj, tx, ty = projection(ab, 5000, 256, 192, seed=2)
    ref = ab.sort_projection(proj["tiles_touched"], proj["rect"], proj["depth"], tx, ty)
    P = len(ref[1])
    tiles, values, ranges, pairs = call(torch, _lib, proj, tx, ty, P - 1, torch.cuda.Stream())
    assert pairs == P
    assert (tiles == np.uint32(0xFFFFFFF9)).all() and (values == np.uint32(0xFFFFFFF9)).all()
    assert not ranges.any()


def test_capacity_zero_counts_only(env):
    """capacity 0 is a count-only call: it succeeds, reports the pair total and writes no pair."""
    torch, ab, _lib = env
    proj, tx, ty = projection(ab, 4000, 192, 128, seed=6)
    ref = ab.sort_projection(proj["tiles_touched"], proj["rect"], proj["depth"], tx, ty)
    for _ in range(2):
        tiles, values, ranges, pairs = call(torch, _lib, proj, tx, ty, 0, torch.cuda.Stream())
        assert pairs == len(ref[1]) > 0
        assert (tiles == np.uint32(0xFFFFFFF9)).all() and (values == np.uint32(0xFFFFFFF9)).all()
        assert not ranges.any()


def test_refuses_oversize_and_bad_rectangles(env):
    torch, ab, _lib = env
    P = ctypes.c_void_p
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    n = _lib.NOALLOC_MAX_GAUSSIANS + 1
    assert _lib.lib.aniso_b200_sort_projection_noalloc(n, P(d.data_ptr()), P(d.data_ptr()), P(d.data_ptr()), 4, 4,
                                                       P(d.data_ptr()), P(d.data_ptr()), 16, P(d.data_ptr()),
                                                       P(d.data_ptr()), None) == _lib.ERR_ARGUMENT
    proj, tx, ty = projection(ab, 2000, 128, 96, seed=3)
    bad = dict(proj)
    bad["rect"] = proj["rect"].copy()
    vis = np.nonzero(proj["tiles_touched"])[0]
    bad["rect"][vis[0], 2] = tx + 5  # x1 outside the grid
    tiles, values, ranges, pairs = call(torch, _lib, bad, tx, ty, 1 << 16, torch.cuda.Stream())
    assert pairs == 0xFFFFFFFFFFFFFFFF
    assert (tiles == np.uint32(0xFFFFFFF9)).all() and not ranges.any()
