"""Runner for oracle/_ref/step_<model>_<n>/ref_step: the reference's own dynamics of the Strang step
(dyn_rate_calc, diffusion_pos, ssa_transport or ssa_substep_1 + optical depth + ssa_substep_2,
compiled from the GameDev tree by oracle/ref/Makefile against a generated model header with
N_P = n).  TEST INFRASTRUCTURE ONLY: it pins the B200 dynamics against the reference's CUDA build;
absent where the reference tree was not mounted at build time."""

from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parents[1] / "_ref"
RNG_BYTES = 48  # curandState (XORWOW)


def binary(model: str, n: int) -> Path:
    return REF_DIR / f"step_{model}_{n}" / "ref_step"


def available(model: str, n: int) -> bool:
    return binary(model, n).exists()


def run(model: str, particles: np.ndarray, seed: int, steps: int, total_dust_mass: float, clock_sim: float = 0.0,
        clock_out: float = 0.0, timeout: float = 600):
    """-> (particles [n, 8] after `steps` dynamics steps, rng states [n, 48] uint8, info with the
    steps' dt and the final clocks)."""
    p = np.ascontiguousarray(particles, dtype=np.float64).reshape(-1, 8)
    n = len(p)
    with tempfile.TemporaryDirectory() as d:
        src, dst = Path(d) / "in.bin", Path(d) / "out.bin"
        with open(src, "wb") as f:
            np.array([n], dtype=np.int32).tofile(f)
            p.tofile(f)
        args = [str(binary(model, n)), str(src), str(dst), str(int(seed)), str(int(steps)),
                repr(float(total_dust_mass)), repr(float(clock_sim)), repr(float(clock_out))]
        r = subprocess.run(args, capture_output=True, text=True, timeout=timeout, cwd=d)
        if r.returncode != 0:
            raise RuntimeError(f"ref_step failed ({r.returncode}): {r.stderr.strip()[-2000:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        raw = np.fromfile(dst, dtype=np.uint8)
        out = raw[4:4 + 64 * n].view(np.float64).reshape(n, 8).copy()
        rng = raw[4 + 64 * n:4 + 64 * n + RNG_BYTES * n].reshape(n, RNG_BYTES).copy()
        return out, rng, info
