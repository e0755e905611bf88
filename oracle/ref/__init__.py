"""Runners and the build recipe for the reference's own code, compiled from the GameDev source tree
where it lies into oracle/_ref.  TEST INFRASTRUCTURE ONLY: the checker, never the product.

REFERENCE_ROOT is the one setting that says where that tree lies on the machine that builds the
checker; the environment variable GD_REFERENCE_ROOT overrides it.  Machines that only run the
checker (the GPU box) never read the tree: the compiled programs travel in oracle/_ref."""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

REFERENCE_ROOT = Path(os.environ.get("GD_REFERENCE_ROOT", "/root/reference"))
HERE = Path(__file__).resolve().parent


def present() -> bool:
    """True where the GameDev source tree can be read (the reference builds need it)."""
    return (REFERENCE_ROOT / "inc" / "swarm").is_dir()


def build(jobs: int = 1) -> None:
    """Compile every reference build of oracle/ref/Makefile into oracle/_ref (incremental)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE), f"-j{jobs}", f"REF={REFERENCE_ROOT}"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle/_ref build failed:\n{r.stdout}\n{r.stderr}")
