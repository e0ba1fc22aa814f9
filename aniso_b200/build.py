"""Builds the in-tree CUDA library aniso_b200/libaniso_b200.so for sm_100a (B200) only.

    python aniso_b200/build.py            # incremental (runs without importing the package)
    python aniso_b200/build.py --force    # rebuild everything

Each csrc/*.cu file is compiled separately (in parallel) with -O3, IEEE division and square root
(no --use_fast_math: the projection must round like the reference kernel built without it),
-lineinfo for ncu source correlation, and -Xptxas -v, whose register / spill / shared-memory
report is written to _build/ptxas.txt. csrc/peaks/peaks.cu becomes libaniso_b200_peaks.so, the
ex2 / FMA throughput probe whose rates are the blend's compute-roofline denominators (the
renderer does not link it). The GpuRenderer shim (shim/gpu_render_shim.cpp) is built
by oracle/Makefile's `dropin` target, against the reference's headers.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libaniso_b200.so")
PEAKS_SRC = os.path.join(CSRC, "peaks", "peaks.cu")
PEAKS_LIB = os.path.join(PKG, "libaniso_b200_peaks.so")
NVCC = os.environ.get("NVCC", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", os.path.join(ROOT, "include")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, headers, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and not _newer(obj, [src] + headers):
        return obj, ""
    cmd = [NVCC] + GENCODE + FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stdout + r.stderr))
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                     + glob.glob(os.path.join(ROOT, "include", "*.h")))
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, headers, force), sources))
    objs = [o for o, _ in results]
    logs = [l for _, l in results if l]
    if logs:
        with open(os.path.join(BUILD, "ptxas.txt"), "w") as f:
            f.write("\n".join(logs))
        if verbose:
            print("\n".join(logs))
    if force or _newer(LIB, objs):
        cmd = [NVCC] + GENCODE + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stdout + r.stderr))
    if force or _newer(PEAKS_LIB, [PEAKS_SRC]):
        cmd = [NVCC] + GENCODE + ["-O3", "-Xcompiler", "-fPIC", "-shared", PEAKS_SRC, "-o", PEAKS_LIB, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (PEAKS_SRC, r.stdout + r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
