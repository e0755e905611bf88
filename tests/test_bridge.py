"""The drop-in bridge (mod/gd_bridge/gd_bridge.cuh) compiled the way a GameDev model directory
compiles it: the model's const_defs.cuh, the reference's gpu.cuh, -DCOLLISION -DMULTISIZE, linked
against libgd_b200.  The program prints the gd_config the bridge derives from the model's
constexprs; it must equal the configuration the library is benchmarked with.  Needs the reference
tree (for gpu.cuh) and nvcc; runs without a GPU."""

import json
import re
import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
from oracle.ref import REFERENCE_ROOT as REF  # noqa: E402

PROGRAM = r"""
#include <const_defs.cuh>
#include <gd_bridge.cuh>
int main() {
    gd_config c = gd_bridge_config();
    int wedge = -1;
    gd_wedge_info(&c, &wedge, nullptr, nullptr);
    std::printf("{\"n_p\": %d, \"n_k\": %d, \"n_x\": %d, \"n_z\": %d, \"coag_kernel\": %d, \"search\": %d, "
                "\"G\": %.17g, \"y_max\": %.17g, \"sigma_0\": %.17g, \"stokes_0\": %.17g, \"v_frag\": %.17g, "
                "\"col_bath_max\": %.17g, \"init_smin\": %.17g, \"code_unit\": %d, \"alpha\": %.17g, "
                "\"x_min\": %.17g, \"x_max\": %.17g, \"x_wedge\": %d, \"gd_wedge\": %d}\n",
                N_P, c.n_k, c.n_x, c.n_z, c.coag_kernel, c.search, c.G, c.y_max, c.sigma_0, c.stokes_0,
                c.v_frag, c.col_bath_max, c.init_smin, c.code_unit, c.alpha, c.x_min, c.x_max,
                static_cast<int>(X_WEDGE), wedge);
    return 0;
}
"""


@pytest.mark.parametrize("model", ["c0_plain_small", "c1_multisize_2d", "c3_learned_3d", "w0_wedge_3d",
                                   "w1_narrow_2d"])
def test_bridge_maps_model_constants(gd, tmp_path, model):
    if not (REF / "inc" / "gpu.cuh").exists():
        pytest.skip("reference tree not mounted (gpu.cuh)")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    src = tmp_path / "bridge_main.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "bridge_main"
    # the model's own flags (flags.mk GPU_FLAGS) and its search, as the reference build sets them
    mk = (ROOT / "mod" / model / "flags.mk").read_text()
    flags = re.findall(r"^GPU_FLAGS \+= (-D\S+)", mk, flags=re.M)
    search = "-DCOLLISION_" + re.search(r"^COLLISION_SEARCH := (\w+)", mk, flags=re.M).group(1).upper()
    cmd = [nvcc, "-std=c++17", *flags, "-DGAMEDEV_CUDA", search,
           "-I", str(ROOT / "mod" / model), "-I", str(ROOT / "mod" / "gd_bridge"), "-I", str(ROOT / "include"),
           "-I", str(REF / "inc"), "-I", str(REF / "inc" / "swarm"),
           str(src), "-o", str(exe), "-L", str(ROOT / "gamedev_b200"), "-lgd_b200",
           "-Xlinker", f"-rpath={ROOT / 'gamedev_b200'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = json.loads(out)
    from gamedev_b200 import workloads

    cfg = workloads.config(model)
    assert got["n_p"] == workloads.CONFIGS[model]["n"]
    for key in ("n_k", "n_x", "n_z", "coag_kernel", "search", "code_unit"):
        assert got[key] == getattr(cfg, key), key
    for key in ("G", "y_max", "sigma_0", "stokes_0", "v_frag", "col_bath_max", "init_smin", "alpha", "x_min",
                "x_max"):
        assert got[key] == getattr(cfg, key), key
    # the library's wedge decision for the bridged configuration is the model's own X_WEDGE
    assert got["gd_wedge"] == got["x_wedge"] == int(model.startswith("w"))
