"""The differentiable path at the forward+backward workload itself: 2.2M Gaussians (30x8x30 box),
1280x720, SH degree 3, L2 loss against the image of the perturbed scene (means + N(0, 0.01), SH DC
+ N(0, 0.05)), gradients of all 59 raw parameters through the torch.autograd.Function -- against
the FP64 oracle at full size (needs a GPU):

* FP64 central differences (h = 1e-4) of the whole-image loss on 256 randomly sampled parameters
  of visible Gaussians, stratified over the five groups; a draw where the renderer takes different
  branches at +h and -h (the loss has a jump or a kink inside [-h, h]) is redrawn and counted;
* the FP64 adjoint of the whole loss given the same dL/dimage, every gradient of every Gaussian;
* the forward image against the FP64 image.

Bar: <= 1e-3 relative error per parameter group, rel = ||g_gpu - g_ref||_2 / ||g_ref||_2.
"""
import json
import os

import numpy as np
import pytest

import oracle
from aniso_b200 import scenes
from oracle import gradcheck

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

REL_TOL = 1e-3


@pytest.fixture(scope="module")
def case():
    import torch

    from aniso_b200.autograd import rasterize

    raws, camsets = scenes.config(3)
    raw, cam = raws[0], camsets[0][0]
    params = gradcheck.raw_param_arrays(raw)
    with torch.no_grad():
        tparams = [torch.tensor(p, device="cuda") for p in gradcheck.raw_param_arrays(scenes.perturbed_target(raw))]
        target_t = rasterize(*tparams, cam)
    ts = [torch.tensor(p, device="cuda", requires_grad=True) for p in params]
    img = rasterize(*ts, cam)
    ((img - target_t) ** 2).sum().backward()
    grads = [t.grad.cpu().numpy().astype(np.float64) for t in ts]
    image = img.detach().cpu().numpy().astype(np.float64)
    target = target_t.cpu().numpy()
    big = oracle.Restatement().big_frame([p.astype(np.float64) for p in params], cam)
    live = np.nonzero(np.abs(grads[0]).sum(1) > 0)[0]
    return {"cam": cam, "grads": grads, "image": image, "target": target, "big": big, "live": live, "n": raw.n}


def report(name, data):
    """Per-group figures go to stdout and, on a GPU box, beside the test logs."""
    print(name, json.dumps(data, indent=1))
    out = os.environ.get("ANISO_B200_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, name + ".json"), "w") as f:
            json.dump(data, f, indent=1)


def test_config3_forward_matches_fp64(case):
    cam = case["cam"]
    ref = case["big"].image(0, 0, cam.width, cam.height)
    err = float(np.abs(case["image"] - ref).max())
    report("config3_forward", {"max_abs": err})
    assert err < 2e-3, err


def test_config3_finite_differences(case):
    res = gradcheck.fd_check(case["big"], case["target"], case["grads"], case["live"], samples=256, step=1e-4)
    report("config3_fd", res)
    for name in gradcheck.GROUPS:
        assert res[name]["samples"] >= 51
        assert res[name]["rel_err"] <= REL_TOL, (name, res[name])


def test_config3_adjoint_every_gradient(case):
    """dL/dimage = 2 (image - target) as the GPU backward received it, through the FP64 adjoint."""
    res = gradcheck.window_check(case["big"], 0, 0, 2 * (case["image"] - case["target"]), case["grads"])
    report("config3_adjoint", res)
    for name in gradcheck.GROUPS:
        assert res[name]["gaussians"] > 100, (name, res[name])
        assert res[name]["rel_err"] <= REL_TOL, (name, res[name])
