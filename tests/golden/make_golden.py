"""Generates the golden fixtures of tests/golden/ from the REFERENCE itself: its CPU renderer,
loader and SH code compiled from its own sources by oracle/Makefile (oracle/_ref/
libaniso_ref_cpu.so), run on seeded inputs in this container.

    make -C oracle reference && python tests/golden/make_golden.py

Writes reference_cpu.npz (small arrays) and reference_cpu.json (image hashes and counts of the
larger cases). The tests check the oracle's C restatement, and through it the GPU path, against
these files, so the oracle stays pinned where the reference cannot be built (the GPU box).
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import kat  # noqa: E402
import oracle  # noqa: E402
from aniso_b200 import scenes  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ref = oracle.ReferenceCPU()
    arrays, meta = {}, {}

    # Known-answer scenes of test_render.cpp, full images.
    for name, make in [("kat_single", kat.kat_single), ("kat_front_back", kat.kat_front_back),
                       ("kat_behind", kat.kat_behind)]:
        g, sh, deg = make()
        img, st = ref.render(g, sh, deg, kat.kat_camera())
        arrays[name + "_image"] = img
        meta[name] = {"visible": st["visible"], "tile_pairs": st["tile_pairs"]}

    # A small degree-3 cloud: image, per-splat projection, SH colour and activation.
    g, sh, deg = kat.random_cloud(1500, seed=21)
    cam = kat.gpu_test_camera(160, 120)
    img, st = ref.render(g, sh, deg, cam)
    splats, radius, alive = ref.make_splats(g, sh, deg, cam)
    arrays.update(cloud_image=img, cloud_splats=splats, cloud_radius=radius, cloud_alive=alive.astype(np.uint8))
    # Inputs are regenerated from their seeds by the tests; their hashes catch generator drift.
    meta["cloud"] = {"visible": st["visible"], "tile_pairs": st["tile_pairs"], "width": 160, "height": 120,
                     "inputs_sha256": sha(g) + sha(sh)}
    for d, s in [(0, 1.0), (1, 0.7), (2, 1.3)]:
        im, _ = ref.render(g, sh, deg, cam, d, s)
        meta["cloud_deg%d_scale%g" % (d, s)] = {"sha256": sha(im)}

    dirs = np.random.default_rng(4).normal(size=(64, 3)).astype(np.float32)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True).astype(np.float32)
    sh1 = np.random.default_rng(5).normal(0, 0.5, size=48).astype(np.float32)
    arrays["sh_dirs"] = dirs
    arrays["sh_coeffs"] = sh1
    arrays["sh_colors"] = np.stack([np.stack([ref.sh_color(sh1, 3, d, deg_) for deg_ in range(4)]) for d in dirs])

    raw = scenes.make_raw_scene(200, (-1, -1, 2), (1, 1, 4), seed=9)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "s.ply")
        scenes.write_ply(path, raw)
        ag, ash, adeg = ref.load_ply(path)
    arrays.update(act_gauss=ag, act_sh=ash)
    meta["activation"] = {"inputs_sha256": sha(raw.xyz) + sha(raw.f_rest) + sha(raw.rot), "degree": adeg}

    # Working-size scenes: image hashes and counts (the images themselves are too large to keep).
    for k in (1, 2):
        scs, cams = scenes.config(k)
        gk, shk = oracle.Restatement().activate(scs[0])
        cam0 = cams[0][0]
        im, st = ref.render(gk, shk, 3, cam0)
        meta["config%d_view0" % k] = {"sha256": sha(im), "visible": st["visible"], "tile_pairs": st["tile_pairs"],
                                      "mean": float(im.mean())}
        arrays["config%d_view0_crop" % k] = im[100:164, 200:264].copy()

    np.savez_compressed(os.path.join(HERE, "reference_cpu.npz"), **arrays)
    with open(os.path.join(HERE, "reference_cpu.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", sorted(arrays), sorted(meta))


if __name__ == "__main__":
    main()
