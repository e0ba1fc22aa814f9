"""Hand-built scenes of the reference's known-answer tests, as activated arrays.

* tests/test_render.cpp:20-73 -- one round Gaussian (analytic centre pixel), a front Gaussian
  hiding a back one listed first, a Gaussian behind the camera.
* tests/test_gpu_render.cpp:17-58 -- a camera with f = 0.8 w and a random cloud of rotated,
  stretched Gaussians with degree-3 colour in front of it (drawn here with numpy's PCG64; the
  reference draws with std::mt19937(7), the distributions are the same).
"""
import numpy as np

from aniso_b200 import scenes

SH_C0 = np.float32(0.28209479177387814)


def kat_camera():
    """64x64, f = 64, principal point at the centre, identity pose (test_render.cpp:22-28)."""
    return scenes.Camera(64, 64, 64.0, 64.0, 32.0, 32.0, np.eye(3), np.zeros(3), "kat")


def gpu_test_camera(w, h):
    """test_gpu_render.cpp:17-23."""
    return scenes.Camera(w, h, 0.8 * w, 0.8 * w, w / 2.0, h / 2.0, np.eye(3), np.zeros(3), "gpu_test")


def _add(gs, shs, pos, scale, opacity, rgb):
    """test_render.cpp:31-38: a round Gaussian whose DC colour gives rgb; degree 0."""
    g = np.zeros(11, np.float32)
    g[0:3] = pos
    g[3:6] = scale
    g[6] = 1.0
    g[10] = opacity
    gs.append(g)
    shs.append(np.array([(np.float32(v) - np.float32(0.5)) / SH_C0 for v in rgb], np.float32))


def kat_single():
    gs, shs = [], []
    _add(gs, shs, (0, 0, 4), 0.2, 0.8, (1.0, 0.0, 0.0))
    return np.stack(gs), np.stack(shs), 0


def kat_front_back():
    gs, shs = [], []
    _add(gs, shs, (0, 0, 8), 0.5, 0.99, (0.0, 0.0, 1.0))  # blue, behind
    _add(gs, shs, (0, 0, 4), 0.2, 0.99, (0.0, 1.0, 0.0))  # green, in front; listed second
    return np.stack(gs), np.stack(shs), 0


def kat_behind():
    gs, shs = [], []
    _add(gs, shs, (0, 0, -4), 0.5, 0.99, (1.0, 1.0, 1.0))
    return np.stack(gs), np.stack(shs), 0


def random_cloud(n, seed=7):
    """The distributions of test_gpu_render.cpp:41-58, activated, SH degree 3."""
    rng = np.random.default_rng(seed)
    u = lambda *s: rng.uniform(-1, 1, size=s).astype(np.float32)
    p01 = lambda *s: rng.uniform(0, 1, size=s).astype(np.float32)
    g = np.zeros((n, 11), np.float32)
    g[:, 0] = u(n) * 2
    g[:, 1] = u(n) * 1.2
    g[:, 2] = 3 + p01(n) * 4
    g[:, 3] = 0.02 + 0.1 * p01(n)
    g[:, 4] = 0.02 + 0.05 * p01(n)
    g[:, 5] = 0.01 + 0.03 * p01(n)
    q = u(n, 4)
    q /= np.sqrt((q * q).sum(1, keepdims=True)).astype(np.float32)
    g[:, 6:10] = q
    g[:, 10] = 0.2 + 0.8 * p01(n)
    sh = np.concatenate([u(n, 3) * 1.5, u(n, 45) * 0.15], axis=1).astype(np.float32)
    return g, sh, 3
