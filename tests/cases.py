"""Seeded small swarms for parity tests, covering the edge-case groups of the reference's KNN suite
(val/swarm/mod/test_knn: equal distances, coincident points, radius boundary, fewer than K,
split planes, inactive filter) with inputs of this project's own making."""

from __future__ import annotations

import math

import numpy as np

from gamedev_b200 import workloads


def code_unit_config(gd, n_k=16, three_d=True, radial_only=False, h_search=1.0, coag_kernel=0):
    """A small code-unit model in the reference's default domain (const_defs.cuh:30-51)."""
    cfg = gd.default_config()
    cfg.n_k = n_k
    cfg.h_search = h_search
    cfg.coag_kernel = coag_kernel
    if radial_only:
        cfg.n_x, cfg.n_z = 1, 1
    elif three_d:
        cfg.n_z = 16
        cfg.z_min, cfg.z_max = 0.5 * math.pi - 0.3, 0.5 * math.pi + 0.3
    return cfg


def random_swarm(cfg, n, seed, inactive_frac=0.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros((n, 8))
    p[:, 0] = rng.uniform(-math.pi, math.pi, n)
    p[:, 1] = rng.uniform(cfg.y_min, cfg.y_max, n)
    if cfg.n_z > 1:
        p[:, 2] = 0.5 * math.pi + rng.normal(0.0, 0.05, n)
    else:
        p[:, 2] = 0.5 * math.pi
    p[:, 3] = np.sqrt(p[:, 1])
    p[:, 6] = np.exp(rng.uniform(math.log(1e-2), math.log(1.0), n))
    p[:, 7] = 1.0 / p[:, 6] ** 3
    if inactive_frac > 0:
        k = int(n * inactive_frac)
        sel = rng.choice(n, k, replace=False)
        p[sel[: k // 2], 1] = cfg.y_max + rng.uniform(0.0, 0.5, k // 2)  # outside [Y_MIN, Y_MAX)
        p[sel[k // 2 :], 1] = cfg.y_min * rng.uniform(0.5, 0.99, k - k // 2)
    return p


def coincident_swarm(cfg, n, seed):
    """Groups of identical positions: ties at d^2 = 0 and at every other distance."""
    p = random_swarm(cfg, n, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    src = rng.integers(0, n, n // 3)
    dst = rng.integers(0, n, n // 3)
    p[dst, :3] = p[src, :3]
    return p


def lattice_swarm(cfg, side, seed):
    """Sites on a regular azimuth x radius (x polar) lattice: many exactly equal distances and
    sites lying on candidate split planes."""
    xs = np.linspace(-math.pi, math.pi, side, endpoint=False)
    ys = np.linspace(cfg.y_min, cfg.y_max, side, endpoint=False)
    zs = (np.linspace(cfg.z_min, cfg.z_max, 4, endpoint=False) if cfg.n_z > 1 else np.array([0.5 * math.pi]))
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    n = X.size
    p = np.zeros((n, 8))
    p[:, 0], p[:, 1], p[:, 2] = X.ravel(), Y.ravel(), Z.ravel()
    p[:, 3] = np.sqrt(p[:, 1])
    p[:, 6] = 0.1
    p[:, 7] = 1.0
    rng = np.random.Generator(np.random.PCG64(seed))
    return p[rng.permutation(n)]


def small_cases(gd):
    cases = []
    cfg = code_unit_config(gd, n_k=32)
    cases.append(("random_3d_k32", cfg, random_swarm(cfg, 3000, 11)))
    cfg = code_unit_config(gd, n_k=16, three_d=False)
    cases.append(("random_2d_k16", cfg, random_swarm(cfg, 2500, 12)))
    cfg = code_unit_config(gd, n_k=8, radial_only=True)
    cases.append(("radial_only_k8", cfg, random_swarm(cfg, 1500, 13)))
    cfg = code_unit_config(gd, n_k=24)
    cases.append(("coincident_k24", cfg, coincident_swarm(cfg, 2000, 14)))
    cfg = code_unit_config(gd, n_k=20)
    cases.append(("lattice_3d_k20", cfg, lattice_swarm(cfg, 24, 15)))
    cfg = code_unit_config(gd, n_k=12, three_d=False)
    cases.append(("lattice_2d_k12", cfg, lattice_swarm(cfg, 40, 16)))
    cfg = code_unit_config(gd, n_k=64, h_search=0.02)
    cases.append(("radius_bound_fewer_than_k", cfg, random_swarm(cfg, 3000, 17)))
    cfg = code_unit_config(gd, n_k=32)
    cases.append(("inactive_filter", cfg, random_swarm(cfg, 3000, 18, inactive_frac=0.2)))
    cfg = code_unit_config(gd, n_k=200)
    cases.append(("k200_reference_default", cfg, random_swarm(cfg, 1200, 19)))
    cfg = code_unit_config(gd, n_k=256)
    cases.append(("k256_more_than_active", cfg, random_swarm(cfg, 150, 20)))
    cfg = workloads.config("c0_plain_small")
    cases.append(("c0_physical_units_k32", cfg, workloads.particles("c0_plain_small", n=4000)))
    return cases
