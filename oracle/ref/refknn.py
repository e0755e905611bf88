"""Runner for oracle/_ref/ref_knn: the reference's own CUDA KD search (kdtree builder, index heap
and traversal, compiled from the GameDev tree by oracle/ref/Makefile) over given sites, driven as
col_cache_get drives it (inc/swarm/_col_cache.cuh:15-71).  TEST INFRASTRUCTURE ONLY: it pins the
B200 search against the reference's CUDA build and times that build; absent where the reference
tree was not mounted at build time."""

from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

BIN = Path(__file__).resolve().parents[1] / "_ref" / "ref_knn"


def available() -> bool:
    return BIN.exists()


def _write_input(path: Path, site4, q, active, k: int):
    n = len(q)
    with open(path, "wb") as f:
        np.array([n, k], dtype=np.int32).tofile(f)
        np.ascontiguousarray(site4, dtype=np.float32).tofile(f)
        np.ascontiguousarray(q, dtype=np.float32).tofile(f)
        np.ascontiguousarray(active, dtype=np.uint8).tofile(f)


def run(site4, q, active, k: int, repeats: int = 0, outputs: bool = True, timeout: float = 600):
    """-> (codes [n][k] int32 in heap order, d2 [n][k] float32, info dict); codes/d2 are None when
    outputs is False (timing only)."""
    n = len(q)
    with tempfile.TemporaryDirectory() as d:
        src, dst = Path(d) / "in.bin", Path(d) / "out.bin"
        _write_input(src, site4, q, active, k)
        r = subprocess.run([str(BIN), str(src), str(dst) if outputs else "-", str(repeats)],
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_knn failed ({r.returncode}): {r.stderr.strip()}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        if not outputs:
            return None, None, info
        raw = np.fromfile(dst, dtype=np.int32)
        codes = raw[: n * k].reshape(n, k)
        d2 = raw[n * k:].view(np.float32).reshape(n, k)
        return codes, d2, info


def canonical(codes, d2):
    """Rows of a heap-ordered cache sorted ascending by (float_bits(d2), code), empty slots last:
    the order the B200 search writes.  Returns (codes, d2, kth) with kth the largest kept d2 (0 for
    an empty row), as col_cache_get feeds _get_ball_measure."""
    valid = codes >= 0
    key = (d2.view(np.uint32).astype(np.uint64) << np.uint64(32)) | codes.astype(np.uint32).astype(np.uint64)
    key = np.where(valid, key, np.uint64(0xFFFFFFFFFFFFFFFF))
    order = np.argsort(key, axis=1, kind="stable")
    c = np.take_along_axis(codes, order, axis=1)
    s = np.take_along_axis(d2, order, axis=1)
    kth = np.where(valid, d2, np.float32(0)).max(axis=1)
    return c, s, kth
