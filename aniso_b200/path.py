"""`aniso path` on the B200: a camera path rendered in batches and streamed as raw RGB frames.

    python -m aniso_b200.path <scene.ply> <path.txt> <WxH> <hfov-degrees> [--sh-degree D] [--batch N]

Same input and output as the reference's command (main.cpp:206-250): one frame per line of the path
file ("px py pz  fx fy fz  ux uy uz [splat_scale]": position, forward, up in world space), 8-bit RGB
rows top to bottom with no header, to stdout, a summary on stderr. Where the reference renders and
copies one frame at a time with two host syncs each, this renders up to N consecutive frames (same
splat scale) as one batch replayed from a CUDA graph into device memory, and copies each batch to
a pinned host buffer on a second stream while the next batch renders (two buffers in turn), so
rendering, the copy back and the write to stdout overlap.
"""
from __future__ import annotations

import math
import sys
import time

import numpy as np

from .renderer import BatchOptions, BatchRenderer, GpuRenderer
from .scenes import Camera


def _norm(v):
    v = np.asarray(v, np.float32)
    l = np.sqrt(np.float32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), dtype=np.float32)
    return np.array([v[0] / l, v[1] / l, v[2] / l], np.float32)


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], np.float32)


def pose_camera(position, forward, up, width: int, height: int, hfov_deg: float, name: str = "") -> Camera:
    """poseCamera (main.cpp:176-199): rows right, down, forward from float vectors; focal from the
    horizontal field of view in double; t = -R p summed in float."""
    p = np.asarray(position, np.float32)
    f = _norm(forward)
    r = _norm(_cross(f, np.asarray(up, np.float32)))
    d = _cross(f, r)
    rows = [r, d, f]
    fx = 0.5 * width / math.tan(hfov_deg * 3.14159265358979 / 360.0)
    R = np.array([[float(x) for x in row] for row in rows], np.float64)
    t = np.array([float(np.float32(-(np.float32(np.float32(row[0] * p[0]) + np.float32(row[1] * p[1]))
                                       + np.float32(row[2] * p[2])))) for row in rows], np.float64)
    return Camera(width, height, fx, fx, width / 2.0, height / 2.0, R, t, name)


def read_path(path_file):
    """(position, forward, up, splat_scale) per non-comment line, as main.cpp:212-222 reads it."""
    poses = []
    with open(path_file) as f:
        for line in f:
            line = line.rstrip("\n")
            if not line or line.startswith("#"):
                continue
            w = line.split()
            if len(w) < 9:
                raise ValueError("bad path line: " + line)
            v = [np.float32(float(x)) for x in w[:9]]
            scale = np.float32(float(w[9])) if len(w) > 9 else np.float32(1.0)
            poses.append((v[0:3], v[3:6], v[6:9], float(scale)))
    return poses


def stream(renderer: GpuRenderer, poses, width: int, height: int, hfov_deg: float, out, sh_degree: int = 3,
           batch: int = 16, use_graph: bool = True) -> int:
    """Renders every pose and writes its RGB frame to the binary file `out`; returns the frame count."""
    import torch

    frame_bytes = width * height * 3
    render_stream = torch.cuda.Stream()
    copy_stream = torch.cuda.Stream()
    dev = [torch.empty((batch, height, width, 3), dtype=torch.uint8, device="cuda") for _ in range(2)]
    host = [torch.empty((batch, height, width, 3), dtype=torch.uint8).pin_memory() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    batches = {}  # (frames, splat scale) -> BatchRenderer, so each shape records its graph once

    groups, k = [], 0
    while k < len(poses):
        j = k + 1
        while j < len(poses) and j - k < batch and poses[j][3] == poses[k][3]:
            j += 1
        groups.append((k, j))
        k = j

    pending = None  # (buffer, frames) copied back but not yet written
    used = [False, False]
    for g, (a, b) in enumerate(groups):
        buf = g % 2
        key = (b - a, poses[a][3])
        if key not in batches:
            batches[key] = BatchRenderer([renderer], [0] * (b - a),
                                         BatchOptions(sh_degree, poses[a][3], (16, 16), 256, use_graph))
        cams = [pose_camera(*poses[i][:3], width, height, hfov_deg) for i in range(a, b)]
        # The device buffer is free once its previous copy back has run.
        if used[buf]:
            render_stream.wait_event(done[buf])
        used[buf] = True
        batches[key].render_device(cams, [dev[buf][i].data_ptr() for i in range(b - a)], render_stream.cuda_stream)
        rendered = torch.cuda.Event()
        rendered.record(render_stream)
        copy_stream.wait_event(rendered)
        with torch.cuda.stream(copy_stream):
            host[buf][: b - a].copy_(dev[buf][: b - a], non_blocking=True)
        done[buf].record(copy_stream)
        if pending is not None:  # write the previous batch while this one renders and copies
            pb, pn = pending
            done[pb].synchronize()
            out.write(memoryview(host[pb].numpy()).cast("B")[: pn * frame_bytes])
        pending = (buf, b - a)
    if pending is not None:
        pb, pn = pending
        done[pb].synchronize()
        out.write(memoryview(host[pb].numpy()).cast("B")[: pn * frame_bytes])
    out.flush()
    for br in batches.values():
        br.sync()  # reports a pair-capacity overflow of any batch
    return len(poses)


def main(argv=None) -> int:
    args = list(sys.argv[1:] if argv is None else argv)
    sh_degree, batch = 3, 16
    for flag in ("--sh-degree", "--batch"):
        if flag in args:
            k = args.index(flag)
            value = int(args[k + 1])
            del args[k:k + 2]
            if flag == "--sh-degree":
                sh_degree = value
            else:
                batch = value
    if len(args) != 4:
        sys.stderr.write("usage: python -m aniso_b200.path <scene.ply> <path.txt> <WxH> <hfov-degrees> "
                         "[--sh-degree 0..3] [--batch N]   (raw RGB to stdout)\n")
        return 2
    ply, path_file, size, hfov = args
    width, height = (int(x) for x in size.lower().split("x"))
    renderer = GpuRenderer.from_ply(ply)
    poses = read_path(path_file)
    t0 = time.perf_counter()
    n = stream(renderer, poses, width, height, float(hfov), sys.stdout.buffer, sh_degree, batch)
    s = time.perf_counter() - t0
    sys.stderr.write("rendered %d frames at %dx%d on the B200 in %.1f s (%.2f ms per frame, including output)\n"
                     % (n, width, height, s, 1000.0 * s / max(1, n)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
