"""aniso_b200_scene_load_ply: the reference loader's header rules and messages (CPU), and on the GPU
the device de-interleave + activation against the same raw values uploaded by
aniso_b200_scene_create_raw and against the reference loader + CPU renderer."""
import os

import numpy as np
import pytest

import oracle
from aniso_b200 import scenes
from conftest import cuda_available


def write_ply(path, columns, names, fmt="binary_little_endian", n=None, truncate=0, extra_element=None):
    """A PLY with the given float columns in the given property order."""
    data = np.stack(columns, 1).astype("<f4")
    n = data.shape[0] if n is None else n
    with open(path, "wb") as f:
        f.write(b"ply\nformat %s 1.0\n" % fmt.encode())
        if extra_element:
            f.write(extra_element.encode())
        f.write(b"element vertex %d\n" % n)
        for nm in names:
            f.write(b"property float %s\n" % nm.encode())
        f.write(b"end_header\n")
        blob = data.tobytes()
        f.write(blob[:len(blob) - truncate])


def raw_columns(raw):
    cols = {"x": raw.xyz[:, 0], "y": raw.xyz[:, 1], "z": raw.xyz[:, 2], "opacity": raw.opacity}
    for k in range(3):
        cols["f_dc_%d" % k] = raw.f_dc[:, k]
        cols["scale_%d" % k] = raw.scale[:, k]
    for k in range(4):
        cols["rot_%d" % k] = raw.rot[:, k]
    for k in range(raw.f_rest.shape[1]):
        cols["f_rest_%d" % k] = raw.f_rest[:, k]
    return cols


def load_status(path):
    import ctypes

    from aniso_b200 import _lib

    h = ctypes.c_void_p()
    rc = _lib.lib.aniso_b200_scene_load_ply(os.fsencode(path), ctypes.byref(h))
    if rc == _lib.OK:
        _lib.lib.aniso_b200_scene_destroy(h)
    return rc, _lib.last_error()


def test_header_errors_are_the_reference_loaders(tmp_path):
    from aniso_b200 import _lib

    raw = scenes.make_raw_scene(10, (-1, -1, 2), (1, 1, 4), seed=1)
    cols = raw_columns(raw)
    names = list(cols)
    p = str(tmp_path / "a.ply")
    open(p, "wb").write(b"not a ply\n")
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": not a PLY file")
    write_ply(p, [cols[k] for k in names], names, fmt="ascii")
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": only binary_little_endian PLY is supported, got ascii")
    write_ply(p, [cols[k] for k in names if k != "rot_2"], [k for k in names if k != "rot_2"])
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": missing property 'rot_2'")
    write_ply(p, [cols[k] for k in names if k != "f_rest_44"], [k for k in names if k != "f_rest_44"])
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": 44 f_rest properties do not match any SH degree")
    write_ply(p, [cols[k] for k in names], names, truncate=8)
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": file is shorter than the header promises (10 Gaussians)")
    write_ply(p, [cols[k] for k in names], names, extra_element="element face 3\n")
    assert load_status(p) == (_lib.ERR_ARGUMENT, p + ": unexpected element 'face'")
    assert load_status(str(tmp_path / "missing.ply")) == (_lib.ERR_ARGUMENT, str(tmp_path / "missing.ply") + ": cannot open")
    write_ply(p, [cols[k] for k in names], names)
    rc, msg = load_status(p)
    assert rc == (_lib.OK if cuda_available() else _lib.ERR_NO_DEVICE), msg


@pytest.mark.gpu
def test_device_ingest_equals_raw_upload_and_reference_loader(tmp_path):
    import aniso_b200 as ab

    raw = scenes.make_raw_scene(20000, (-2, -1.5, 3), (2, 1.5, 8), seed=5)
    cols = raw_columns(raw)
    rng = np.random.default_rng(0)
    names = list(cols) + ["nx", "ny"]
    cols["nx"] = rng.normal(size=raw.n).astype(np.float32)
    cols["ny"] = np.zeros(raw.n, np.float32)
    order = [names[k] for k in rng.permutation(len(names))]  # any property order
    p = str(tmp_path / "scene.ply")
    write_ply(p, [cols[k] for k in order], order)
    cam = scenes.Camera(320, 240, 260.0, 260.0, 160.0, 120.0, np.eye(3), np.zeros(3))

    r_ply = ab.GpuRenderer.from_ply(p)
    r_raw = ab.GpuRenderer.from_raw(raw)
    assert (r_ply.n, r_ply.sh_degree) == (raw.n, 3)
    a, b = r_ply.debug_projection(cam), r_raw.debug_projection(cam)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    img = r_ply.render(cam)
    np.testing.assert_array_equal(img, r_raw.render(cam))
    if oracle.ReferenceCPU.available():
        ref = oracle.ReferenceCPU()
        g, sh, deg = ref.load_ply(p)
        cpu, _ = ref.render(g, sh, deg, cam)
    else:
        g, sh = scenes.activate(raw)
        cpu, _ = oracle.Restatement().render(g, sh, 3, cam)
    d = int(np.abs(img.astype(np.int32) - cpu.astype(np.int32)).max())
    assert d <= 2 and oracle.psnr(img, cpu) >= 75.0
