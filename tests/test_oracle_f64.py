"""The FP64 gradient oracle's full-size form (BigFrame: depth-ordered 8x8-tile lists and local
queries) against its whole-image form on small scenes, on the CPU. The full-size form is what the
gradient checks at the 2.2M-Gaussian workload use, where the whole-image form is out of reach."""
import numpy as np
import pytest

import oracle
from aniso_b200 import scenes


def small_case(n=160, seed=3):
    rng = np.random.default_rng(seed)
    params = [np.stack([rng.uniform(-1, 1, n), rng.uniform(-0.7, 0.7, n), rng.uniform(3, 6, n)], 1),
              rng.normal(-2.6, 0.4, (n, 3)), rng.normal(0, 1, (n, 4)), rng.normal(0, 1, n),
              rng.normal(0, 0.3, (n, 16, 3))]
    params = [a.astype(np.float32).astype(np.float64) for a in params]
    cam = scenes.Camera(72, 56, 60.0, 60.0, 36.0, 28.0, np.eye(3), np.zeros(3))
    target = rng.uniform(0, 1, (56, 72, 3)).astype(np.float32)
    return params, cam, target


def test_window_image_equals_whole_image_render():
    params, cam, _ = small_case()
    R = oracle.Restatement()
    full = R.train_forward_f64(params, cam)
    big = R.big_frame(params, cam)
    np.testing.assert_array_equal(big.image(0, 0, cam.width, cam.height), full)
    np.testing.assert_array_equal(big.image(9, 5, 30, 20), full[5:25, 9:39])
    v, p = big.counts()
    assert 0 < v <= 160 and p >= v


def test_window_adjoint_equals_whole_image_adjoint():
    params, cam, target = small_case()
    R = oracle.Restatement()
    img = R.train_forward_f64(params, cam)
    grad = 2 * (img - target)
    full = R.train_backward_f64(params, cam, grad)
    big = R.big_frame(params, cam)
    for a, b in zip(big.adjoint(0, 0, grad), full):
        np.testing.assert_array_equal(a, b)
    # a window: the adjoint of the loss restricted to it
    mask = np.zeros_like(grad)
    mask[10:40, 20:60] = 1
    win = R.train_backward_f64(params, cam, grad * mask)
    for a, b in zip(big.adjoint(20, 10, grad[10:40, 20:60]), win):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("group,comp", [(0, 0), (0, 2), (1, 1), (2, 3), (3, 0), (4, 0), (4, 29)])
def test_local_central_difference_equals_whole_image_difference(group, comp):
    params, cam, target = small_case()
    R = oracle.Restatement()
    big = R.big_frame(params, cam)
    gref = R.train_backward_f64(params, cam, 2 * (R.train_forward_f64(params, cam) - target))
    live = np.nonzero(np.abs(gref[0]).sum(1) > 0)[0]
    loss = lambda P: ((R.train_forward_f64(P, cam) - target.astype(np.float64)) ** 2).sum()
    h = 1e-4
    for i in live[:6]:
        idx = (int(i),) + np.unravel_index(comp, params[group].shape[1:])
        Pp = [a.copy() for a in params]
        Pm = [a.copy() for a in params]
        Pp[group][idx] += h
        Pm[group][idx] -= h
        whole = (loss(Pp) - loss(Pm)) / (2 * h)
        local, smooth, px = big.fd(target, i, group, comp, h)
        assert px > 0
        assert abs(local - whole) <= 1e-7 * max(1.0, abs(whole)), (i, local, whole)


def test_branch_flip_is_flagged():
    """A step that moves a splat's alpha across the 1/255 cut somewhere is reported as not smooth,
    and a tiny step of the same parameter as smooth."""
    params, cam, target = small_case()
    R = oracle.Restatement()
    big = R.big_frame(params, cam)
    gref = R.train_backward_f64(params, cam, 2 * (R.train_forward_f64(params, cam) - target))
    live = np.nonzero(np.abs(gref[0]).sum(1) > 0)[0]
    flags_big = [big.fd(target, i, 0, 0, 0.2)[1] for i in live[:20]]   # a large move of the mean
    flags_tiny = [big.fd(target, i, 0, 0, 1e-9)[1] for i in live[:20]]
    assert not all(flags_big)
    assert sum(flags_tiny) >= 18
