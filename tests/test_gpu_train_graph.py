"""The training batch replayed from CUDA graphs (rasterize_batch with use_graph, the default) gives
the same bytes as the same batch launched plainly and as the views differentiated one by one, on
every launch shape, step after step while the parameter tensors move and the cameras change
(needs a GPU)."""
import numpy as np
import pytest

from aniso_b200 import BatchOptions, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def params_of(torch, n, seed):
    rng = np.random.default_rng(seed)
    arrs = [np.stack([rng.uniform(-1.5, 1.5, n), rng.uniform(-1, 1, n), rng.uniform(3, 7, n)], 1),
            rng.normal(-3.0, 0.4, (n, 3)), rng.normal(0, 1, (n, 4)), rng.normal(0, 1, n),
            rng.normal(0, 0.3, (n, 16, 3))]
    return [torch.tensor(a, dtype=torch.float32, device="cuda") for a in arrs]


def cameras(shift):
    return [scenes.Camera(160, 120, 130.0, 130.0, 80.0, 60.0, np.eye(3), np.array([shift, 0.0, 0.0])),
            scenes.Camera(200, 112, 150.0, 150.0, 100.0, 56.0, np.eye(3), np.array([-shift, 0.05, 0.0])),
            scenes.Camera(96, 96, 80.0, 80.0, 48.0, 48.0, np.eye(3), np.array([0.0, shift, 0.0]))]


def step(torch, scene_tensors, cams, view_scene, ups, **kw):
    from aniso_b200.autograd import rasterize_batch

    leaves = [[t.detach().clone().requires_grad_(True) for t in s] for s in scene_tensors]
    imgs = rasterize_batch(leaves, cams, view_scene, **kw)
    torch.autograd.backward(imgs, ups)
    torch.cuda.synchronize()
    return [i.detach().cpu().numpy() for i in imgs], [t.grad.cpu().numpy() for g in leaves for t in g]


def per_view(torch, scene_tensors, cams, view_scene, ups):
    from aniso_b200.autograd import rasterize

    leaves = [[t.detach().clone().requires_grad_(True) for t in s] for s in scene_tensors]
    imgs = []
    for c, s, u in zip(cams, view_scene, ups):
        img = rasterize(*leaves[s], c)
        torch.autograd.backward([img], [u])
        imgs.append(img.detach().cpu().numpy())
    torch.cuda.synchronize()
    return imgs, [t.grad.cpu().numpy() for g in leaves for t in g]


def assert_same(a, b, what):
    for x, y in zip(a[0] + a[1], b[0] + b[1]):
        np.testing.assert_array_equal(x, y, err_msg=what)


def test_graph_replays_equal_plain_and_per_view(torch):
    view_scene = [0, 0, 1]
    gen = torch.Generator(device="cuda").manual_seed(9)
    for k in range(3):  # new tensors, new cameras, the same shapes: the recorded graphs replay
        sc = [params_of(torch, 3000, 10 + k), params_of(torch, 1500, 20 + k)]
        cams = cameras(0.05 * k)
        ups = [torch.randn((c.height, c.width, 3), device="cuda", generator=gen) for c in cams]
        g = step(torch, sc, cams, view_scene, ups, use_graph=True)
        p = step(torch, sc, cams, view_scene, ups, use_graph=False)
        v = per_view(torch, sc, cams, view_scene, ups)
        assert_same(g, p, "graph vs plain, step %d" % k)
        assert_same(g, v, "graph vs per view, step %d" % k)
        assert any(x.any() for x in g[1])


@pytest.mark.parametrize("tile,bb,bits", [((8, 8), 128, 8), ((16, 32), 256, 9), ((16, 16), 128, 8)])
def test_every_launch_shape_gives_the_same_step(torch, tile, bb, bits):
    """Every shape renders the same images bit for bit. The gradients are the same sums grouped by
    a different tile grid (each Gaussian adds up one slot per tile it touches), so they agree to
    rounding across shapes, and bit for bit between a recorded graph's replays and plain launches of
    the same shape (and, at 16x16, with the per-view path)."""
    view_scene = [0, 1, 1]
    sc = [params_of(torch, 2500, 31), params_of(torch, 2000, 32)]
    cams = cameras(0.03)
    gen = torch.Generator(device="cuda").manual_seed(5)
    ups = [torch.randn((c.height, c.width, 3), device="cuda", generator=gen) for c in cams]
    ref = per_view(torch, sc, cams, view_scene, ups)
    opt = lambda graph: BatchOptions(3, 1.0, tile, bb, graph, bits)
    plain = step(torch, sc, cams, view_scene, ups, options=opt(False))
    for _ in range(2):  # record, then replay
        got = step(torch, sc, cams, view_scene, ups, options=opt(True))
        assert_same(got, plain, "graph vs plain %s/%d/%d" % (tile, bb, bits))
    for a, b in zip(got[0], ref[0]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(got[1], ref[1]):
        np.testing.assert_allclose(a, b, rtol=1e-4, atol=1e-5 * max(1e-30, float(np.abs(b).max())))
    if tuple(tile) == (16, 16):
        assert_same(got, ref, "16x16 vs per view")


def test_tune_train_picks_a_shape(torch):
    from aniso_b200.autotune import tune_train

    sc = [params_of(torch, 2000, 41), params_of(torch, 1000, 42)]
    report = []
    best = tune_train(sc, cameras(0.02), [0, 0, 1], cache_path=None, report=report, iters=1)
    assert len(report) == 12 and best.use_graph
    assert min(r["ms"] for r in report) == next(r["ms"] for r in report
                                                 if tuple(r["tile"]) == tuple(best.tile) and
                                                 r["blend_batch"] == best.blend_batch and
                                                 r["radix_bits"] == best.radix_bits)
