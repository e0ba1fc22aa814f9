"""The training step around the adjoint (needs a GPU): the fused Adam against torch.optim.Adam, the
densification rules on a crafted state, and a short fit that must lower the loss."""
import numpy as np
import pytest

from aniso_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def random_params(torch, n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = lambda *s, scale=1.0: torch.randn(*s, generator=g, device="cuda") * scale
    means = torch.stack([r(n, scale=1.0), r(n, scale=0.7), r(n).abs() * 2 + 3], 1)
    return {"means": means, "log_scales": r(n, 3, scale=0.4) - 2.6, "quats": r(n, 4),
            "opacity_logits": r(n), "sh": r(n, 16, 3, scale=0.3)}


def test_fused_adam_matches_torch_adam(torch):
    from aniso_b200 import train

    params = random_params(torch, 1000, 0)
    model = train.GaussianModel(params, scene_scale=3.0)
    lrs = {"means": 1e-3, "log_scales": 5e-3, "quats": 1e-3, "opacity_logits": 5e-2, "sh": 2.5e-3}
    ref = {k: params[k].clone().requires_grad_(True) for k in train.NAMES if k != "sh"}
    sh0 = params["sh"][:, :1].clone().requires_grad_(True)
    shn = params["sh"][:, 1:].clone().requires_grad_(True)
    groups = [{"params": [ref[k]], "lr": lrs[k]} for k in ref] + [{"params": [sh0], "lr": lrs["sh"]},
                                                                 {"params": [shn], "lr": lrs["sh"] / 20}]
    opt = torch.optim.Adam(groups, eps=1e-15)
    g = torch.Generator(device="cuda").manual_seed(1)
    for step in range(1, 6):
        grads = {k: torch.randn(model.p[k].shape, generator=g, device="cuda") for k in train.NAMES}
        for k in train.NAMES:
            model.p[k].grad = grads[k].clone()
        for k in ref:
            ref[k].grad = grads[k].clone()
        sh0.grad, shn.grad = grads["sh"][:, :1].clone(), grads["sh"][:, 1:].clone()
        train.adam_step(model, lrs, lrs["sh"] / 20, step)
        opt.step()
    torch.cuda.synchronize()
    for k in ref:
        torch.testing.assert_close(model.p[k].detach(), ref[k].detach(), rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(model.p["sh"].detach(), torch.cat([sh0, shn], 1).detach(), rtol=1e-5, atol=1e-6)


def test_densify_rules(torch):
    from aniso_b200 import train

    n = 10
    params = random_params(torch, n, 2)
    params["log_scales"][:] = np.log(0.01)         # small: <= grow_scale3d * scene_scale = 0.02
    params["log_scales"][5:8] = np.log(0.05)       # large
    params["opacity_logits"][:] = 0.0              # opacity 0.5
    params["opacity_logits"][9] = -8.0             # below prune_opa
    model = train.GaussianModel(params, scene_scale=2.0)
    model.grad2d[:] = torch.tensor([1e-3, 1e-3, 0, 0, 0, 1e-3, 1e-3, 0, 0, 0], device="cuda")
    model.visible[:] = 1.0
    t = train.Trainer(model, total_steps=1000, densify=train.Densify(refine_start=0, refine_every=10))
    t._refine(10)
    # +2 duplicates (0, 1), +2 net from splitting (5, 6), -1 pruned (9)
    assert model.n == n + 2 + 2 - 1
    assert float(model.grad2d.abs().sum()) == 0.0 and float(model.visible.sum()) == 0.0
    for k in train.NAMES:
        assert model.p[k].shape[0] == model.n and model.m[k].shape[0] == model.n


def test_short_fit_lowers_the_loss(torch):
    from aniso_b200 import train
    from aniso_b200.autograd import rasterize

    truth = random_params(torch, 3000, 3)
    cams = [scenes.Camera(128, 96, 110.0, 110.0, 64.0, 48.0, np.eye(3), np.array([0.3 * k - 0.45, 0.0, 0.0]))
            for k in range(4)]
    with torch.no_grad():
        targets = [rasterize(*[truth[k] for k in train.NAMES], c, sh_degree=0) for c in cams]
    start = {k: v.clone() for k, v in truth.items()}
    g = torch.Generator(device="cuda").manual_seed(4)
    start["means"] += torch.randn(start["means"].shape, generator=g, device="cuda") * 0.05
    start["sh"][:, 0] = 0.0
    start["opacity_logits"][:] = -2.0
    model = train.GaussianModel(start, scene_scale=3.0)
    t = train.Trainer(model, total_steps=200, densify=train.Densify(refine_start=60, refine_every=60),
                      sh_degree=0)
    losses = [t.step(cams[k % 4], targets[k % 4]) for k in range(200)]
    assert all(np.isfinite(losses))
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:20]), (losses[:5], losses[-5:])
