"""The drop-in through the reference's model-directory interface, end to end.

oracle/_ref/gamedev_c1_multisize_2d_65536/ holds the reference's whole program (every
src/swarm/*.cu, its main and time loop included) built twice from the GameDev tree by
oracle/ref/Makefile for the same generated model directory (c1 shapes: 2D, Morton search,
coagulation and fragmentation, one output frame):
  * stock/gamedev  as the reference ships it;
  * dropin/gamedev with the model-local swarm_runtime.cu mod/gd_bridge/make_runtime.py writes, whose
                   evolve_collisions lambda and controller reset call libgd_b200 through
                   mod/gd_bridge/gd_bridge.cuh, linked against gamedev_b200/libgd_b200.so.
Both resume from the same injected frame 0 (particle_00000.dat and rngstate_00000.dat, written by
gd_save_checkpoint in the reference's formats) and run one output interval (`gamedev 0`).  Bars on
the frame-1 files they write: positions and velocities byte-identical (a collision-only model
moves no particle), every grain size and count within 1e-12 relative of the stock build's (the
Morton rows are in the same order, so the event chains are the same), represented mass conserved
to 1e-12, and the RNG states identical as streams.
"""

import math
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
MODEL, N = "c1_multisize_2d", 65536
BASE = ROOT / "oracle" / "_ref" / f"gamedev_{MODEL}_{N}"


def _run(binary: Path, workdir: Path):
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = str(ROOT / "gamedev_b200") + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    r = subprocess.run([str(binary), "0"], cwd=workdir, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, (binary, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


def test_dropin_gamedev_equals_stock_gamedev(gd, cuda, tmp_path):
    import torch

    from gamedev_b200 import workloads

    stock, dropin = BASE / "stock" / "gamedev", BASE / "dropin" / "gamedev"
    if not (stock.exists() and dropin.exists()):
        pytest.fail(f"{BASE} is missing: build the checker first (__graft_entry__.build)")
    cfg = workloads.config(MODEL)
    p = workloads.particles(MODEL, n=N)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(N, seed=1)
    outs = {}
    for label, binary in (("stock", stock), ("dropin", dropin)):
        work = tmp_path / label
        (work / "out").mkdir(parents=True)
        gd.save_checkpoint(cfg, str(work / "out") + "/", 0, dp, rng, save_max=1)
        if label == "stock":
            # frame 0 as the programs read it (the file stores linear speeds: the conversion back
            # rounds the angular momenta)
            frame0 = torch.empty_like(dp)
            gd.load_checkpoint(cfg, str(work / "out") + "/", 0, frame0, None, save_max=1)
            p0 = frame0.cpu().numpy()
        _run(binary, work)
        part = torch.empty_like(dp)
        st = torch.empty_like(rng)
        gd.load_checkpoint(cfg, str(work / "out") + "/", 1, part, st, save_max=1)
        torch.cuda.synchronize()
        outs[label] = (part.cpu().numpy(), gd.rng_uniforms(st, N, 4).cpu().numpy())
    (a, ua), (b, ub) = outs["stock"], outs["dropin"]
    assert np.array_equal(a[:, :6].view(np.uint64), b[:, :6].view(np.uint64))
    assert np.array_equal(a[:, :6].view(np.uint64), p0[:, :6].view(np.uint64))
    for col in (6, 7):
        rel = np.abs(b[:, col] - a[:, col]) / np.abs(a[:, col])
        assert rel.max() <= 1e-12, (col, float(rel.max()), int(np.argmax(rel)))
    changed = int((a[:, 6] != p[:, 6]).sum())
    assert changed > N // 100, changed  # the interval holds collisions
    m0 = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    m1 = float((b[:, 7] * math.pi * b[:, 6] ** 3 / 6.0).sum())
    assert abs(m1 - m0) <= 1e-12 * m0
    assert np.array_equal(ua, ub)
