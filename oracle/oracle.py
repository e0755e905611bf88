"""ctypes binding of the CPU oracle (oracle/_build/libgd_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU arms,
never by the gamedev_b200 package.  The oracle restates the reference algorithm on the host; see
gd_oracle.h for the reference file:line each function follows.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgd_oracle.so"

_lib = None


def build() -> Path:
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        P = C.c_void_p
        lib.gdo_site_init.restype = C.c_int
        lib.gdo_site_init.argtypes = [P, P, C.c_int, P, P, P]
        lib.gdo_knn_brute.restype = None
        lib.gdo_knn_brute.argtypes = [C.c_int, P, P, P, C.c_int, P, P, C.c_int]
        lib.gdo_knn_brute_images.restype = None
        lib.gdo_knn_brute_images.argtypes = [C.c_int, C.c_int, P, P, P, C.c_int, C.c_float, C.c_float, P, P,
                                             C.c_int]
        lib.gdo_morton_ghosts.restype = None
        lib.gdo_morton_ghosts.argtypes = [C.c_int, P, P, C.c_float, C.c_float, C.c_float, P, P]
        lib.gdo_knn_kdtree.restype = None
        lib.gdo_knn_kdtree.argtypes = [C.c_int, P, P, P, C.c_int, P, P, C.c_int, C.c_int, C.c_int]
        lib.gdo_kdtree_build.restype = P
        lib.gdo_kdtree_build.argtypes = [C.c_int, P, P]
        lib.gdo_kdtree_query.restype = None
        lib.gdo_kdtree_query.argtypes = [P, C.c_int, P, P, C.c_int, P, P, C.c_int, C.c_int, C.c_int]
        lib.gdo_kdtree_free.restype = None
        lib.gdo_kdtree_free.argtypes = [P]
        lib.gdo_ball_measure.restype = None
        lib.gdo_ball_measure.argtypes = [P, P, C.c_int, P, P, P]
        lib.gdo_space_bin.restype = None
        lib.gdo_space_bin.argtypes = [P, P, C.c_int, P]
        _extend(lib)
        _lib = lib
    return _lib


def _extend(lib):
    """Bind the collision-operator restatement when present."""
    P = C.c_void_p
    if hasattr(lib, "gdo_env"):
        lib.gdo_env.restype = None
        lib.gdo_env.argtypes = [P, C.c_double, C.c_double, P]
    for name in ("gdo_pair_speed_cached", "gdo_pair_speed_direct"):
        if hasattr(lib, name):
            getattr(lib, name).restype = C.c_double
    if hasattr(lib, "gdo_pair_speed_cached"):
        lib.gdo_pair_speed_cached.argtypes = [P, P, C.c_double, C.c_double]
        lib.gdo_pair_speed_direct.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_double]
    if hasattr(lib, "gdo_outcome_moments"):
        lib.gdo_outcome_moments.restype = C.c_double
        lib.gdo_outcome_moments.argtypes = [P, C.c_double, C.c_double, C.c_int, P]
        lib.gdo_sample_outcome.restype = C.c_double
        lib.gdo_sample_outcome.argtypes = [P, C.c_double, C.c_double, C.c_int, C.c_double]
    if hasattr(lib, "gdo_pair_rate"):
        lib.gdo_pair_rate.restype = C.c_double
        lib.gdo_pair_rate.argtypes = [P] + [C.c_double] * 9 + [P]
    if hasattr(lib, "gdo_bath_rate"):
        lib.gdo_bath_rate.restype = None
        lib.gdo_bath_rate.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_double, P, P, P, P, C.c_int]
    if hasattr(lib, "gdo_chain_owner"):
        lib.gdo_chain_owner.restype = C.c_int
        lib.gdo_chain_owner.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_double, C.c_double, P, P, C.c_int, P, P]


def _p(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _cfg_ptr(cfg):
    return C.byref(cfg)


def site_init(cfg, particles: np.ndarray):
    """col_site_init restated: returns (site4 float32 [n,4], q float32 [n], active uint8 [n], bad)."""
    p = np.ascontiguousarray(particles).view(np.float64).reshape(-1, 8)
    n = p.shape[0]
    site4 = np.zeros((n, 4), np.float32)
    q = np.zeros(n, np.float32)
    active = np.zeros(n, np.uint8)
    bad = load().gdo_site_init(_cfg_ptr(cfg), _p(p), n, _p(site4), _p(q), _p(active))
    return site4, q, active, bad


def knn_brute(site4, q, active, k: int, threads: int | None = None):
    n = site4.shape[0]
    codes = np.empty((n, k), np.int32)
    d2 = np.empty((n, k), np.float32)
    load().gdo_knn_brute(n, _p(site4), _p(q), _p(active), k, _p(codes), _p(d2), threads or os.cpu_count())
    return codes, d2


def knn_brute_images(site4, n: int, q, active, k: int, image_dist_min: float, q_dedup: float = -1.0,
                     threads: int | None = None):
    """Top-K of owners 0..n-1 over every site of `site4` (wedge images included), with the duplicate
    image dedup of the reference heap (gdo_knn_brute_images)."""
    site4 = np.ascontiguousarray(site4, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    active = np.ascontiguousarray(active, np.uint8)
    codes = np.empty((n, k), np.int32)
    d2 = np.empty((n, k), np.float32)
    load().gdo_knn_brute_images(n, site4.shape[0], _p(site4), _p(q), _p(active), k, float(image_dist_min),
                                float(q_dedup), _p(codes), _p(d2), threads or os.cpu_count())
    return codes, d2


def morton_ghosts(site4, posx, q_max: float, x_min: float, x_max: float):
    """The Morton ghost rule over the n physical sites `site4[:n]` (gdo_morton_ghosts): returns
    keep (n, 2), columns image 1 and image 2, and each decision's relative margin from q_max."""
    site4 = np.ascontiguousarray(site4, np.float32)
    posx = np.ascontiguousarray(posx, np.float32)
    n = posx.shape[0]
    keep = np.empty((n, 2), np.uint8)
    margin = np.empty((n, 2), np.float64)
    load().gdo_morton_ghosts(n, _p(site4), _p(posx), float(q_max), float(np.float32(x_min)),
                             float(np.float32(x_max)), _p(keep), _p(margin))
    return keep.astype(bool), margin


def knn_kdtree(site4, q, active, k: int, threads: int | None = None, first: int = 0, count: int = -1):
    n = site4.shape[0]
    codes = np.full((n, k), -1, np.int32)
    d2 = np.zeros((n, k), np.float32)
    load().gdo_knn_kdtree(n, _p(site4), _p(q), _p(active), k, _p(codes), _p(d2), threads or os.cpu_count(),
                          first, count)
    return codes, d2


class KdTree:
    """The oracle KD tree kept alive between queries (for timing the CPU baseline)."""

    def __init__(self, site4, active):
        self.site4 = np.ascontiguousarray(site4, np.float32)
        self.active = np.ascontiguousarray(active, np.uint8)
        self.n = self.site4.shape[0]
        self.h = load().gdo_kdtree_build(self.n, _p(self.site4), _p(self.active))

    def query(self, q, k, codes, d2=None, threads=None, first=0, count=-1):
        load().gdo_kdtree_query(self.h, self.n, _p(q), _p(self.active), k, _p(codes), _p(d2),
                                threads or os.cpu_count(), first, count)

    def close(self):
        if self.h:
            load().gdo_kdtree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kth_from_rows(codes, d2):
    """Largest kept d^2 per row (0 for an empty row)."""
    valid = codes >= 0
    out = np.where(valid, d2, 0.0).max(axis=1) if codes.shape[1] else np.zeros(codes.shape[0])
    return out.astype(np.float32)


def ball_measure(cfg, particles, active, kth):
    p = np.ascontiguousarray(particles).view(np.float64).reshape(-1, 8)
    n = p.shape[0]
    out = np.empty(n, np.float64)
    act = np.ascontiguousarray(active, np.uint8)
    kth = np.ascontiguousarray(kth, np.float32)
    load().gdo_ball_measure(_cfg_ptr(cfg), _p(p), n, _p(act), _p(kth), _p(out))
    return out


def space_bin(cfg, particles):
    p = np.ascontiguousarray(particles).view(np.float64).reshape(-1, 8)
    out = np.empty(p.shape[0], np.int32)
    load().gdo_space_bin(_cfg_ptr(cfg), _p(p), p.shape[0], _p(out))
    return out


# ---- collision operator restatement ------------------------------------------------------------
def env(cfg, y, z):
    out = np.zeros(8, np.float64)
    load().gdo_env(_cfg_ptr(cfg), float(y), float(z), _p(out))
    return out


def pair_speed(cfg, y, z, size_i, size_j):
    """Pair speed as the operator evaluates it: cached environment in physical units, direct
    formula in code units."""
    lib = load()
    if not cfg.code_unit and not cfg.const_st:
        e = env(cfg, y, z)
        return lib.gdo_pair_speed_cached(_cfg_ptr(cfg), _p(e), float(size_i), float(size_j))
    return lib.gdo_pair_speed_direct(_cfg_ptr(cfg), float(y), float(z), float(size_i), float(size_j))


def pair_rate(cfg, yi, zi, yj, zj, size_i, size_j, numr_j, lambda0, measure):
    """(rate / measure, pair speed) of one owner-partner pair."""
    v = C.c_double(0.0)
    r = load().gdo_pair_rate(_cfg_ptr(cfg), float(yi), float(zi), float(yj), float(zj), float(size_i),
                             float(size_j), float(numr_j), float(lambda0), float(measure), C.byref(v))
    return r, v.value


def outcome_moments(cfg, si, sj, high):
    out = np.zeros(3, np.float64)
    f = load().gdo_outcome_moments(_cfg_ptr(cfg), float(si), float(sj), int(bool(high)), _p(out))
    return f, out[0], out[1], out[2]


def sample_outcome(cfg, si, sj, high, u):
    return load().gdo_sample_outcome(_cfg_ptr(cfg), float(si), float(sj), int(bool(high)), float(u))


def bath_rate(cfg, particles, codes, measure, active, size_old, numr_old, lambda0, threads=None):
    p = np.ascontiguousarray(particles).view(np.float64).reshape(-1, 8)
    n = p.shape[0]
    cached = np.zeros((n, 4), np.float64)
    rate = np.zeros(n)
    change = np.zeros(n)
    second = np.zeros(n)
    # keep every converted array alive across the call
    codes = np.ascontiguousarray(codes, np.int32)
    measure = np.ascontiguousarray(measure, np.float64)
    active = np.ascontiguousarray(active, np.uint8)
    size_old = np.ascontiguousarray(size_old, np.float64)
    numr_old = np.ascontiguousarray(numr_old, np.float64)
    load().gdo_bath_rate(_cfg_ptr(cfg), n, _p(p), _p(codes), _p(measure), _p(active), _p(size_old), _p(numr_old),
                         float(lambda0), _p(cached), _p(rate), _p(change), _p(second), threads or os.cpu_count())
    return cached, rate, change, second


def chain_owner(cfg, i, particles, codes, measure, active, size_old, numr_old, lambda0, bath_end, cached4, uniforms):
    """One owner through one bath; returns (error, state[8], uniforms used)."""
    p = np.ascontiguousarray(particles).view(np.float64).reshape(-1, 8)
    state = np.zeros(8, np.float64)
    state[0] = p[i, 6]
    state[1] = p[i, 7]
    used = C.c_int(0)
    u = np.ascontiguousarray(uniforms, np.float64)
    codes = np.ascontiguousarray(codes, np.int32)
    measure = np.ascontiguousarray(measure, np.float64)
    active = np.ascontiguousarray(active, np.uint8)
    size_old = np.ascontiguousarray(size_old, np.float64)
    numr_old = np.ascontiguousarray(numr_old, np.float64)
    cached4 = np.ascontiguousarray(cached4, np.float64)
    err = load().gdo_chain_owner(_cfg_ptr(cfg), int(i), _p(p), _p(codes), _p(measure), _p(active), _p(size_old),
                                 _p(numr_old), float(lambda0), float(bath_end), _p(cached4), _p(u), len(u),
                                 _p(state), C.byref(used))
    return err, state, used.value
