"""The training path's per-splat block bits drop only splats that could not take part: the
training forward (raw tensors, block bits in the records, the blend's training variant) quantised
to 8 bits equals the plain render of the same raw scene (activated on the device with the same
functions, no block bits) byte for byte, on scenes whose splats range from sub-pixel to hundreds of
pixels, thin and round, near and far (needs a GPU)."""
import numpy as np
import pytest

from aniso_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available()
    return torch


def quantise(img):
    """render.cpp's 8-bit quantisation of a float colour, in fp32: clamp to [0, 1], x 255, + 0.5."""
    c = np.clip(img.astype(np.float32), np.float32(0), np.float32(1))
    return (c * np.float32(255) + np.float32(0.5)).astype(np.uint8)


def tensors(torch, raw):
    n = raw.n
    sh = np.concatenate([raw.f_dc.reshape(n, 1, 3), raw.f_rest.reshape(n, 3, 15).transpose(0, 2, 1)], 1)
    arrs = [raw.xyz, raw.scale, raw.rot, raw.opacity, np.ascontiguousarray(sh)]
    return [torch.tensor(a, dtype=torch.float32, device="cuda") for a in arrs]


CASES = {
    # name: (Gaussians, box lo, box hi, log-scale shift, camera (w, h, f, distance))
    "small_splats": (20000, (-2, -1.5, -2), (2, 1.5, 2), 0.0, (320, 240, 300.0, 6.0)),
    "large_splats": (3000, (-2, -1.5, -2), (2, 1.5, 2), 2.0, (320, 240, 300.0, 6.0)),
    "near_and_wide": (8000, (-3, -2, -3), (3, 2, 3), 1.0, (640, 360, 400.0, 3.5)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_training_forward_equals_plain_render(torch, case):
    from aniso_b200 import GpuRenderer
    from aniso_b200.autograd import rasterize

    n, lo, hi, shift, (w, h, f, dist) = CASES[case]
    raw = scenes.make_raw_scene(n, lo, hi, seed=17)
    raw.scale = (raw.scale + np.float32(shift)).astype(np.float32)  # bigger splats
    cam = scenes.front_camera(w, h, f, dist)
    with torch.no_grad():
        train = rasterize(*tensors(torch, raw), cam).cpu().numpy()
    plain = GpuRenderer.from_raw(raw).render(cam)
    assert plain.any()
    np.testing.assert_array_equal(quantise(train), plain)
