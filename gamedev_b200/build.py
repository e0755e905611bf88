"""Build libgd_b200.so in-tree with nvcc for sm_100a.

The library is the product: hand-written CUDA kernels and the C ABI declared in include/gd_b200.h.
It is compiled straight into this package directory so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libgd_b200.so"
OBJ = PKG / "_build"

SOURCES = ["gd_geometry.cu", "gd_range.cu", "gd_collide.cu", "gd_controller.cu", "gd_radius.cu", "gd_api.cu",
           "gd_batch.cu", "gd_io.cu", "gd_transport.cu", "gd_devctl.cu"]
# The device controller compiles the host controller's arithmetic; without FMA contraction its
# roundings are the host's, so the schedule and baths it picks are the host controller's, bit for bit.
SOURCE_FLAGS = {"gd_devctl.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include")]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgd_b200")
    return exe


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "gd_b200.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = OBJ / (s.stem + ".o")
        objs.append(o)
        if force or ptxas_info or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH, *FLAGS, *SOURCE_FLAGS.get(src, []), "-c", str(s), "-o", str(o)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_info or verbose:
                sys.stdout.write(r.stderr)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
