"""The persistent sort (one cooperative launch with bounded grid barriers, selected by
ANISO_B200_SORT=persistent, read once per process, hence child processes) and the multi-kernel
sort (the default) give the same bytes: sorted pair lists and tile ranges of single views, images of
batches of mixed resolutions and tile shapes (8- and 9-bit tile digits), gradients of the
differentiable path (needs a GPU)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + '/tests')
import kat, torch
import aniso_b200
from aniso_b200 import scenes, BatchRenderer, BatchOptions
from aniso_b200._lib import lib
from aniso_b200.autograd import rasterize
out = {}
# single views: sorted pairs and ranges (large enough for several rounds per CTA)
g, sh, d = kat.random_cloud(60000, seed=17)
r = aniso_b200.GpuRenderer(g, sh, d)
for w, h in ((1280, 720), (333, 217), (1, 1)):
    t, v, rg = r.debug_sorted(kat.gpu_test_camera(w, h))
    out['t%d' % w], out['v%d' % w], out['r%d' % w] = t, v, rg
# a batch: two scenes, views of mixed sizes; 16x32 tiles with 9-bit digits and 8x8 tiles
g2, sh2, d2 = kat.random_cloud(30000, seed=18)
r2 = aniso_b200.GpuRenderer(g2, sh2, d2)
cams = [kat.gpu_test_camera(w, h) for w, h in ((640, 360), (1920, 1080), (320, 240), (1280, 720))]
for name, opt in (('b9', BatchOptions(tile=(16, 32), blend_batch=256, radix_bits=9, use_graph=True)),
                  ('b8', BatchOptions(tile=(8, 8), blend_batch=128, radix_bits=8, use_graph=False))):
    b = BatchRenderer([r, r2], [0, 0, 1, 1], opt)
    outs = [torch.zeros((c.height, c.width, 3), dtype=torch.uint8, device='cuda') for c in cams]
    for _ in range(3):  # the first frames may overflow the pair capacity and grow it
        b.render_device(cams, [o.data_ptr() for o in outs], torch.cuda.current_stream().cuda_stream)
        try:
            b.sync()
        except aniso_b200.AnisoError as e:
            assert 'pair capacity' in str(e)
    for k, o in enumerate(outs):
        out['%s_%d' % (name, k)] = o.cpu().numpy()
# gradients of the differentiable path
rng = np.random.default_rng(3)
n = 5000
P = [np.stack([rng.uniform(-1.5, 1.5, n), rng.uniform(-1, 1, n), rng.uniform(3, 7, n)], 1),
     rng.normal(-3.2, 0.4, (n, 3)), rng.normal(0, 1, (n, 4)), rng.normal(0, 1, n), rng.normal(0, 0.3, (n, 16, 3))]
ts = [torch.tensor(p, dtype=torch.float32, device='cuda', requires_grad=True) for p in P]
img = rasterize(*ts, kat.gpu_test_camera(320, 240))
img.square().sum().backward()
out['img'] = img.detach().cpu().numpy()
for k, t in enumerate(ts):
    out['g%d' % k] = t.grad.cpu().numpy()
np.savez(OUT, **out)
"""


def run_child(tmp_path, mode):
    path = str(tmp_path / ("%s.npz" % mode))
    code = "ROOT = %r\nOUT = %r\n" % (ROOT, path) + CHILD
    env = dict(os.environ)
    if mode == "persistent":
        env["ANISO_B200_SORT"] = "persistent"
    else:
        env.pop("ANISO_B200_SORT", None)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return dict(np.load(path))


def test_persistent_sort_equals_multi_kernel_sort(tmp_path):
    a = run_child(tmp_path, "persistent")
    b = run_child(tmp_path, "default")
    assert set(a) == set(b)
    for key in sorted(a):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    assert a["v1280"].size > 100000 and a["img"].any()
