"""Runner for oracle/_ref/collide_<model>_<n>/ref_collide: the reference's own CUDA collision step
(evolve_collisions glue + evolve_local_collisions and its kernels, compiled from the GameDev tree
by oracle/ref/Makefile against a generated model header with N_P = n).  TEST INFRASTRUCTURE ONLY:
it pins the B200 collision operator against the reference's CUDA build and times it; absent where
the reference tree was not mounted at build time."""

from __future__ import annotations

import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parents[1] / "_ref"


def binary(model: str, n: int, diagnostics: bool = False) -> Path:
    return REF_DIR / f"collide{'_diag' if diagnostics else ''}_{model}_{n}" / "ref_collide"


def available(model: str, n: int, diagnostics: bool = False) -> bool:
    return binary(model, n, diagnostics).exists()


def run(model: str, particles: np.ndarray, seed: int, duration: float, total_dust_mass: float,
        operators: int = 1, timeout: float = 1800, diagnostics: bool = False, neighbours: bool = False,
        records: bool = False, steps: int = 1):
    """-> (particles after `operators` evolve_collisions(duration) calls on one geometry, info).
    With diagnostics (the COL_DIAGNOSTICS build), info["summary"] holds the controller summary the
    reference's save_col_controller wrote, parsed, info["summary_text"] its text, and
    info["operator_log"] the parsed lines of its per-operator log.  With neighbours,
    info["codes"] [n][K] and info["measure"] [n] hold the neighbour cache col_cache_get wrote; with
    records, info["records"] [count][4] float32 holds the search's records (x, y, z, code bits): the
    KD nodes, or the Morton index's points with its periodic ghosts.  With steps > 1 the geometry and
    the operators repeat `steps` times (a swarm step each: GD_REF_STEPS of ref_collide.cu) and
    info["steps"] lists [geometry_ms, operator_ms...] per step; the dumps describe the first step."""
    p = np.ascontiguousarray(particles, dtype=np.float64).reshape(-1, 8)
    n = len(p)
    with tempfile.TemporaryDirectory() as d:
        src, dst = Path(d) / "in.bin", Path(d) / "out.bin"
        with open(src, "wb") as f:
            np.array([n], dtype=np.int32).tofile(f)
            p.tofile(f)
        summary = Path(d) / "summary.json"
        args = [str(binary(model, n, diagnostics)), str(src), str(dst), str(int(seed)), repr(float(duration)),
                repr(float(total_dust_mass)), str(int(operators))]
        if diagnostics:
            args.append(str(summary))
        env = dict(os.environ)
        nb, rb = Path(d) / "neighbours.bin", Path(d) / "records.bin"
        if neighbours:
            env["GD_REF_NEIGHBOURS"] = str(nb)
        if records:
            env["GD_REF_SITES"] = str(rb)
        env["GD_REF_STEPS"] = str(int(steps))
        r = subprocess.run(args, capture_output=True, text=True, timeout=timeout, cwd=d, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"ref_collide failed ({r.returncode}): {r.stderr.strip()[-2000:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        if diagnostics:
            info["summary_text"] = summary.read_text()
            info["summary"] = json.loads(info["summary_text"])
            logs = sorted(Path(d).glob("collision_local_*.jsonl"))
            info["operator_log"] = [json.loads(line) for f in logs for line in f.read_text().splitlines()
                                    if line.strip()]
        if neighbours:
            raw = np.fromfile(nb, dtype=np.uint8)
            n_p, k = raw[:8].view(np.int32)
            info["codes"] = raw[8:8 + 4 * n_p * k].view(np.int32).reshape(n_p, k).copy()
            info["measure"] = raw[8 + 4 * n_p * k:].view(np.float64).copy()
        if records:
            raw = np.fromfile(rb, dtype=np.uint8)
            count = int(raw[:4].view(np.int32)[0])
            info["records"] = raw[4:4 + 16 * count].view(np.float32).reshape(count, 4).copy()
        raw = np.fromfile(dst, dtype=np.uint8)
        out = raw[4:].view(np.float64).reshape(n, 8).copy()
        return out, info
