"""Seeded synthetic 3DGS scenes and COLMAP pinhole cameras.

The public Tanks&Temples *train* scene and the licence-restricted Kitchen scene behind the
reference's published timings (README.md:28-29) are not available, so every workload is a seeded
synthetic scene with the distributions below, drawn with numpy's PCG64 ``default_rng(seed)``,
columns in this order: xyz, f_dc, f_rest, opacity, scale, rot.

* xyz     uniform in an axis-aligned box
* f_dc    N(0, 0.5)
* f_rest  N(0, 0.05), 45 values, channel-major as in the 3DGS PLY layout
* opacity logit ~ N(0, 1.5)
* scale   log-scale ~ N(-4.0, 0.5)
* rot     normalise(N(0, 1)^4), w first

Scenes are kept in the raw (optimizer) form a PLY stores; :func:`activate` applies the
conversions of the reference loader (ply_loader.cpp:124-138): exp(scale), sigmoid(opacity),
normalised quaternion, and the f_rest reorder from channel-major to [coefficient][channel].

Cameras follow aniso::Camera (camera.h:16-26): world-to-camera R (row-major) and t in double,
fx, fy, cx, cy in pixels, COLMAP's axes (x right, y down, z forward).
"""
from __future__ import annotations

import dataclasses
import os
import struct

import numpy as np

SH_C0 = 0.28209479177387814


@dataclasses.dataclass
class RawScene:
    """Raw per-Gaussian values in the 3DGS PLY layout (all float32)."""

    xyz: np.ndarray      # (N, 3)
    f_dc: np.ndarray     # (N, 3)
    f_rest: np.ndarray   # (N, 3 * (K - 1)) channel-major
    opacity: np.ndarray  # (N,) logit
    scale: np.ndarray    # (N, 3) log
    rot: np.ndarray      # (N, 4) w, x, y, z

    @property
    def n(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def sh_degree(self) -> int:
        rest = self.f_rest.shape[1] // 3
        for d in range(5):
            if (d + 1) ** 2 - 1 == rest:
                return d
        raise ValueError("f_rest width matches no SH degree")

    def sh_coeffs(self) -> np.ndarray:
        """SH as (N, K, 3), [coefficient][channel] (the reorder of ply_loader.cpp:132-138)."""
        n = self.n
        k = (self.sh_degree + 1) ** 2
        out = np.empty((n, k, 3), np.float32)
        out[:, 0, :] = self.f_dc
        if k > 1:
            out[:, 1:, :] = self.f_rest.reshape(n, 3, k - 1).transpose(0, 2, 1)
        return out


@dataclasses.dataclass
class Camera:
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    R: np.ndarray  # (3, 3) float64, world to camera, row-major
    t: np.ndarray  # (3,) float64
    name: str = ""

    def packed(self) -> np.ndarray:
        """16 doubles: R[9] row-major, t[3], fx, fy, cx, cy (the C-ABI camera layout)."""
        return np.concatenate([self.R.reshape(9), self.t.reshape(3),
                               [self.fx, self.fy, self.cx, self.cy]]).astype(np.float64)

    def centre(self) -> np.ndarray:
        return -(self.R.T @ self.t)


def make_raw_scene(n: int, lo, hi, seed: int, sh_degree: int = 3) -> RawScene:
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    xyz = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    f_dc = rng.normal(0.0, 0.5, size=(n, 3)).astype(np.float32)
    rest = 3 * ((sh_degree + 1) ** 2 - 1)
    f_rest = rng.normal(0.0, 0.05, size=(n, rest)).astype(np.float32)
    opacity = rng.normal(0.0, 1.5, size=n).astype(np.float32)
    scale = rng.normal(-4.0, 0.5, size=(n, 3)).astype(np.float32)
    rot = rng.normal(0.0, 1.0, size=(n, 4))
    rot /= np.linalg.norm(rot, axis=1, keepdims=True)
    return RawScene(xyz, f_dc, f_rest, opacity, scale, rot.astype(np.float32))


def activate(raw: RawScene):
    """(gauss (N, 11), sh (N, K*3)) activated the way the reference loader does.

    gauss columns: x, y, z, sx, sy, sz, qw, qx, qy, qz, opacity -- the memory layout of
    std::vector<aniso::Gaussian> (gaussian.h:21-26). Computed in float32; numpy's exp may differ
    from the C library's expf in the last bit, so parity tests activate through the oracle's C
    restatement instead and feed the same arrays to every renderer.
    """
    n = raw.n
    g = np.empty((n, 11), np.float32)
    g[:, 0:3] = raw.xyz
    g[:, 3:6] = np.exp(raw.scale.astype(np.float32))
    q = raw.rot.astype(np.float32)
    norm = np.sqrt((q * q).sum(axis=1, dtype=np.float32)).astype(np.float32)
    safe = np.where(norm > 0, norm, np.float32(1))
    qn = (q / safe[:, None]).astype(np.float32)
    qn[norm <= 0] = np.array([1, 0, 0, 0], np.float32)
    g[:, 6:10] = qn
    g[:, 10] = (np.float32(1) / (np.float32(1) + np.exp(-raw.opacity.astype(np.float32)))).astype(np.float32)
    return g, raw.sh_coeffs().reshape(n, -1).copy()


def look_at(position, target, width, height, f, up=(0.0, -1.0, 0.0), name="") -> Camera:
    """A camera at `position` aimed at `target`, rows (right, down, forward) as in the
    reference CLI's poseCamera (main.cpp:179-202); world -y is up."""
    p = np.asarray(position, np.float64)
    fwd = np.asarray(target, np.float64) - p
    fwd /= np.linalg.norm(fwd)
    r = np.cross(fwd, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    d = np.cross(fwd, r)
    R = np.stack([r, d, fwd])
    t = -R @ p
    return Camera(int(width), int(height), float(f), float(f), width / 2.0, height / 2.0, R, t, name)


def ring_cameras(count, radius, width, height, f, y=0.0):
    """`count` cameras on a horizontal ring around the origin; camera 0 sits at (0, y, -radius)."""
    cams = []
    for k in range(count):
        a = 2.0 * np.pi * k / count
        pos = (radius * np.sin(a), y, -radius * np.cos(a))
        cams.append(look_at(pos, (0.0, 0.0, 0.0), width, height, f, name="ring_%03d" % k))
    return cams


def fibonacci_cameras(count, radius, resolutions, seed, focal_frac=0.9):
    """`count` cameras on a Fibonacci sphere aimed at the origin, resolution drawn per camera."""
    rng = np.random.default_rng(seed)
    pick = rng.integers(len(resolutions), size=count)
    golden = np.pi * (3.0 - np.sqrt(5.0))
    cams = []
    for k in range(count):
        yy = 1.0 - 2.0 * (k + 0.5) / count
        rr = np.sqrt(max(0.0, 1.0 - yy * yy))
        phi = golden * k
        pos = radius * np.array([rr * np.cos(phi), yy, rr * np.sin(phi)])
        w, h = resolutions[pick[k]]
        cams.append(look_at(pos, (0.0, 0.0, 0.0), w, h, focal_frac * w, name="sphere_%03d" % k))
    return cams


def front_camera(width, height, f, distance):
    """The camera at (0, 0, -distance) looking down +z (R = I)."""
    return look_at((0.0, 0.0, -distance), (0.0, 0.0, 0.0), width, height, f, name="front")


# The five workload shapes. Sizes, boxes and seeds as listed; `scale` shrinks N for quick runs.
RESOLUTIONS_4 = [(320, 180), (640, 360), (1280, 720), (1920, 1080)]


def config(k: int, scale: float = 1.0):
    """Returns (list of RawScene, list of list of Camera) for workload k in 1..5."""
    def n_(x):
        return max(1, int(round(x * scale)))

    if k == 1:  # 100k Gaussians, one camera at the origin looking down +z, 640x360, f=500
        s = make_raw_scene(n_(100_000), (-4, -4, 2), (4, 4, 12), seed=0)
        cam = Camera(640, 360, 500.0, 500.0, 320.0, 180.0, np.eye(3), np.zeros(3), "origin")
        return [s], [[cam]]
    if k == 2:  # 740k in a 20x6x20 box, 16 ring cameras radius 8, 1280x720, f=1100
        s = make_raw_scene(n_(740_000), (-10, -3, -10), (10, 3, 10), seed=0)
        return [s], [ring_cameras(16, 8.0, 1280, 720, 1100.0)]
    if k == 3:  # 2.2M in a 30x8x30 box, camera 8 units back looking +z, 1280x720, f=1100
        s = make_raw_scene(n_(2_200_000), (-15, -4, -15), (15, 4, 15), seed=0)
        return [s], [[front_camera(1280, 720, 1100.0, 8.0)]]
    if k == 4:  # 1M in a 20^3 box, 64 Fibonacci-sphere cameras radius 10, mixed resolutions
        s = make_raw_scene(n_(1_000_000), (-10, -10, -10), (10, 10, 10), seed=0)
        return [s], [fibonacci_cameras(64, 10.0, RESOLUTIONS_4, seed=3)]
    if k == 5:  # 8 scenes of uneven size, 4 ring views each, 960x540 / 1280x720 alternating
        sizes = [200_000, 400_000, 700_000, 1_000_000, 1_500_000, 2_000_000, 2_500_000, 3_000_000]
        scenes, cams = [], []
        for i, m in enumerate(sizes):
            scenes.append(make_raw_scene(n_(m), (-15, -4, -15), (15, 4, 15), seed=10 + i))
            views = []
            for v in range(4):
                w, h = (960, 540) if v % 2 == 0 else (1280, 720)
                a = 2.0 * np.pi * v / 4
                pos = (8.0 * np.sin(a), 0.0, -8.0 * np.cos(a))
                views.append(look_at(pos, (0, 0, 0), w, h, 1100.0 * w / 1280.0, name="s%d_v%d" % (i, v)))
            cams.append(views)
        return scenes, cams
    raise ValueError("workload 1..5")


def perturbed_target(raw: RawScene, seed: int = 1) -> RawScene:
    """The fwd+bwd target scene: means + N(0, 0.01), SH DC + N(0, 0.05)."""
    rng = np.random.default_rng(seed)
    xyz = (raw.xyz + rng.normal(0, 0.01, raw.xyz.shape)).astype(np.float32)
    f_dc = (raw.f_dc + rng.normal(0, 0.05, raw.f_dc.shape)).astype(np.float32)
    return RawScene(xyz, f_dc, raw.f_rest, raw.opacity, raw.scale, raw.rot)


# --- files: the 3DGS PLY and COLMAP sparse models (text and binary) -------------------------

def write_ply(path, raw: RawScene):
    """Binary little-endian PLY in the reference 3DGS layout (x y z nx ny nz f_dc f_rest opacity
    scale rot), the layout the reference loader reads (ply_loader.cpp:20-65)."""
    n = raw.n
    cols = [raw.xyz, np.zeros((n, 3), np.float32), raw.f_dc, raw.f_rest, raw.opacity[:, None], raw.scale, raw.rot]
    data = np.concatenate(cols, axis=1).astype("<f4")
    names = (["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
             + ["f_rest_%d" % i for i in range(raw.f_rest.shape[1])]
             + ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"])
    with open(path, "wb") as f:
        f.write(b"ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n)
        for nm in names:
            f.write(b"property float %s\n" % nm.encode())
        f.write(b"end_header\n")
        f.write(data.tobytes())


def read_ply(path) -> RawScene:
    """Reads the layout write_ply writes (any column order, float32 properties only)."""
    with open(path, "rb") as f:
        if f.readline().strip() != b"ply":
            raise ValueError("not a PLY file")
        props, n = [], 0
        while True:
            line = f.readline()
            if not line:
                raise ValueError("header has no end_header")
            w = line.split()
            if not w:
                continue
            if w[0] == b"format" and w[1] != b"binary_little_endian":
                raise ValueError("only binary_little_endian PLY is supported")
            if w[0] == b"element" and w[1] == b"vertex":
                n = int(w[2])
            if w[0] == b"property":
                if w[1] not in (b"float", b"float32"):
                    raise ValueError("non-float property")
                props.append(w[2].decode())
            if w[0] == b"end_header":
                break
        body = np.frombuffer(f.read(n * len(props) * 4), "<f4")
        if body.size != n * len(props):
            raise ValueError("file is shorter than the header promises")
        body = body.reshape(n, len(props))
    col = {p: i for i, p in enumerate(props)}
    rest = 0
    while "f_rest_%d" % rest in col:
        rest += 1
    pick = lambda names: body[:, [col[x] for x in names]].astype(np.float32)
    return RawScene(pick(["x", "y", "z"]), pick(["f_dc_0", "f_dc_1", "f_dc_2"]),
                    pick(["f_rest_%d" % i for i in range(rest)]), pick(["opacity"])[:, 0],
                    pick(["scale_0", "scale_1", "scale_2"]), pick(["rot_0", "rot_1", "rot_2", "rot_3"]))


def _rot_to_quat(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix."""
    m = R
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0:
        s = np.sqrt(tr + 1.0) * 2
        return np.array([0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s])
    if m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = np.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2
        return np.array([(m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s])
    if m[1, 1] > m[2, 2]:
        s = np.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2
        return np.array([(m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s])
    s = np.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2
    return np.array([(m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s])


def write_colmap(folder, cams, binary=True, text=True):
    """COLMAP sparse model, one PINHOLE camera per image: cameras/images .bin (what the reference
    reads, camera.cpp:61-140) and .txt (COLMAP's text format)."""
    os.makedirs(folder, exist_ok=True)
    if binary:
        with open(os.path.join(folder, "cameras.bin"), "wb") as f:
            f.write(struct.pack("<Q", len(cams)))
            for i, c in enumerate(cams):
                f.write(struct.pack("<IiQQ", i + 1, 1, c.width, c.height))
                f.write(struct.pack("<4d", c.fx, c.fy, c.cx, c.cy))
        with open(os.path.join(folder, "images.bin"), "wb") as f:
            f.write(struct.pack("<Q", len(cams)))
            for i, c in enumerate(cams):
                q = _rot_to_quat(c.R)
                f.write(struct.pack("<I", i + 1))
                f.write(struct.pack("<4d", *q))
                f.write(struct.pack("<3d", *c.t))
                f.write(struct.pack("<I", i + 1))
                f.write((c.name or "img_%03d" % i).encode() + b"\0")
                f.write(struct.pack("<Q", 0))
    if text:
        with open(os.path.join(folder, "cameras.txt"), "w") as f:
            f.write("# Camera list with one line of data per camera:\n")
            f.write("#   CAMERA_ID, MODEL, WIDTH, HEIGHT, PARAMS[]\n")
            for i, c in enumerate(cams):
                f.write("%d PINHOLE %d %d %.17g %.17g %.17g %.17g\n" % (i + 1, c.width, c.height, c.fx, c.fy, c.cx, c.cy))
        with open(os.path.join(folder, "images.txt"), "w") as f:
            f.write("# Image list with two lines of data per image:\n")
            f.write("#   IMAGE_ID, QW, QX, QY, QZ, TX, TY, TZ, CAMERA_ID, NAME\n")
            f.write("#   POINTS2D[] as (X, Y, POINT3D_ID)\n")
            for i, c in enumerate(cams):
                q = _rot_to_quat(c.R)
                f.write("%d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %s\n\n"
                        % (i + 1, q[0], q[1], q[2], q[3], c.t[0], c.t[1], c.t[2], i + 1, c.name or "img_%03d" % i))


def read_colmap_text(folder):
    """Reads cameras.txt/images.txt (PINHOLE / SIMPLE_PINHOLE) into Cameras sorted by image name,
    with the same quaternion-to-matrix conversion as camera.cpp:95-101."""
    intr = {}
    with open(os.path.join(folder, "cameras.txt")) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            w = line.split()
            cid, model, width, height = int(w[0]), w[1], int(w[2]), int(w[3])
            p = [float(x) for x in w[4:]]
            if model == "SIMPLE_PINHOLE":
                intr[cid] = (width, height, p[0], p[0], p[1], p[2])
            elif model == "PINHOLE":
                intr[cid] = (width, height, p[0], p[1], p[2], p[3])
            else:
                raise ValueError("camera model %s has lens distortion; undistort the images first" % model)
    cams = []
    with open(os.path.join(folder, "images.txt")) as f:
        lines = [l for l in f if not l.startswith("#")]
    for i in range(0, len(lines), 2):
        w = lines[i].split()
        if not w:
            continue
        qw, qx, qy, qz = (float(x) for x in w[1:5])
        t = np.array([float(x) for x in w[5:8]])
        width, height, fx, fy, cx, cy = intr[int(w[8])]
        nrm = np.sqrt(qw * qw + qx * qx + qy * qy + qz * qz)
        qw, qx, qy, qz = qw / nrm, qx / nrm, qy / nrm, qz / nrm
        R = np.array([[1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)],
                      [2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)],
                      [2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)]])
        cams.append(Camera(width, height, fx, fy, cx, cy, R, t, w[9]))
    cams.sort(key=lambda c: c.name)
    return cams


# COLMAP model ids and their parameter counts (COLMAP's models.h; the table of camera.cpp:57-60).
_COLMAP_PARAMS = [3, 4, 4, 5, 8, 8, 12, 5, 4, 5, 12]


def _quat_to_matrix(qw, qx, qy, qz):
    """camera.cpp:95-101: normalise in double, then the rotation matrix of the unit quaternion."""
    nrm = np.sqrt(qw * qw + qx * qx + qy * qy + qz * qz)
    w, x, y, z = qw / nrm, qx / nrm, qy / nrm, qz / nrm
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def read_colmap_binary(folder):
    """cameras.bin / images.bin as aniso::loadColmapCameras reads them (camera.cpp:61-140): PINHOLE
    and SIMPLE_PINHOLE only, each image's 2D points skipped, Cameras sorted by image name."""
    def take(f, fmt):
        size = struct.calcsize(fmt)
        b = f.read(size)
        if len(b) != size:
            raise ValueError("%s: truncated" % f.name)
        return struct.unpack(fmt, b)

    intr = {}
    with open(os.path.join(folder, "cameras.bin"), "rb") as f:
        (count,) = take(f, "<Q")
        for _ in range(count):
            cid, model, width, height = take(f, "<IiQQ")
            if model < 0 or model >= len(_COLMAP_PARAMS):
                raise ValueError("%s: unknown camera model %d" % (f.name, model))
            p = take(f, "<%dd" % _COLMAP_PARAMS[model])
            if model == 0:
                intr[cid] = (width, height, p[0], p[0], p[1], p[2])
            elif model == 1:
                intr[cid] = (width, height, p[0], p[1], p[2], p[3])
            else:
                raise ValueError("%s: camera model %d has lens distortion; undistort the images first"
                                 % (f.name, model))
    cams = []
    with open(os.path.join(folder, "images.bin"), "rb") as f:
        (count,) = take(f, "<Q")
        for _ in range(count):
            take(f, "<I")
            q = take(f, "<4d")
            t = np.array(take(f, "<3d"))
            (cid,) = take(f, "<I")
            name = bytearray()
            while True:
                ch = f.read(1)
                if not ch:
                    raise ValueError("%s: truncated" % f.name)
                if ch == b"\0":
                    break
                name += ch
            (points,) = take(f, "<Q")
            f.seek(points * 24, os.SEEK_CUR)
            if cid not in intr:
                raise ValueError("%s: image %s refers to a missing camera" % (f.name, name.decode()))
            width, height, fx, fy, cx, cy = intr[cid]
            cams.append(Camera(width, height, fx, fy, cx, cy, _quat_to_matrix(*q), t, name.decode()))
    cams.sort(key=lambda c: c.name)
    return cams


def read_colmap(folder):
    """A COLMAP sparse model in either form: the binary one when cameras.bin is there (what the
    reference reads), else the text one (what the workload descriptions are written in)."""
    if os.path.exists(os.path.join(folder, "cameras.bin")):
        return read_colmap_binary(folder)
    return read_colmap_text(folder)
