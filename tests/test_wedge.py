"""Azimuthal wedges on the host: the periodic-image parameters and the oracle's duplicate-image dedup.

In a wedge (n_x > 1, azimuth shorter than 2 pi) the reference gives every particle two images
rotated by -width and +width (src/swarm/col_site_init.cu:58-76).  An owner whose search ball can
reach two images of one particle (image_dist_min <= 2 q) keeps only the nearer one, by
(d^2 bits, code) (kdtree/index_heap.cuh:118-141; the Morton search's id sort,
morton/morton_query.cuh:18-58 and 62-140, keeps the same one).
"""

import ctypes
import math

import numpy as np
import pytest


def _wedge_sites(n, width, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(1.0, 2.0, n)
    phi = rng.uniform(0.0, width, n)
    base = np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(0.0, 0.05, n)], 1)
    sites = np.zeros((3 * n, 4), np.float32)
    for img, ang in ((0, 0.0), (1, -width), (2, width)):
        c, s = math.cos(ang), math.sin(ang)
        blk = sites[img * n:(img + 1) * n]
        blk[:, 0] = c * base[:, 0] - s * base[:, 1]
        blk[:, 1] = s * base[:, 0] + c * base[:, 1]
        blk[:, 2] = base[:, 2]
        blk[:, 3] = (3 * np.arange(n, dtype=np.int32) + img).view(np.float32)
    return sites


def _first_per_particle(row, k):
    """The first entry of each particle along an ascending row, up to k (the dedup's result)."""
    out, seen = [], set()
    for c in row:
        if c < 0:
            break
        if c // 3 in seen:
            continue
        seen.add(c // 3)
        out.append(c)
        if len(out) == k:
            break
    return out + [-1] * (k - len(out))


def test_oracle_dedup_keeps_the_nearest_image_of_each_particle():
    from oracle import oracle

    n, K, width = 400, 40, 0.05  # a sliver: the K nearest reach across the seams
    sites = _wedge_sites(n, width, seed=11)
    q = np.full(n, 0.4, np.float32)
    active = np.ones(n, np.uint8)
    active[::17] = 0
    # every candidate of every owner, ascending (K = all sites, no dedup)
    all_codes, _ = oracle.knn_brute_images(sites, n, q, active, 3 * n, -1.0)
    # image_dist_min = 0.1 <= 2 q: every owner deduplicates
    codes, d2 = oracle.knn_brute_images(sites, n, q, active, K, 0.1)
    plain, _ = oracle.knn_brute_images(sites, n, q, active, K, -1.0)
    repeats = 0
    for i in range(n):
        if not active[i]:
            assert (codes[i] == -1).all()
            continue
        assert codes[i].tolist() == _first_per_particle(all_codes[i], K), i
        assert plain[i].tolist() == all_codes[i][:K].tolist(), i
        kept = plain[i][plain[i] >= 0] // 3
        repeats += int(len(kept) != len(set(kept.tolist())))
    assert repeats > 0  # the case holds owners that see two images of one particle
    # the Morton search's decision uses the largest q: 2 * 0.01 < 0.1, no owner deduplicates
    morton_off, _ = oracle.knn_brute_images(sites, n, q, active, K, 0.1, q_dedup=0.01)
    assert np.array_equal(morton_off, plain)
    # image_dist_min > 2 q: unique identifiers, the plain top-K
    unique, _ = oracle.knn_brute_images(sites, n, q, active, K, 0.81)
    assert np.array_equal(unique, plain)


def _libm_sinf():
    libm = ctypes.CDLL("libm.so.6")
    libm.sinf.restype = ctypes.c_float
    libm.sinf.argtypes = [ctypes.c_float]
    return lambda x: np.float32(libm.sinf(np.float32(x)))


@pytest.mark.parametrize("workload", ["w0_wedge_3d", "w1_narrow_2d", "w2_wide_3d", "c0_plain_small",
                                      "c1_multisize_2d"])
def test_wedge_info_restates_x_wedge_and_image_dist_min(gd, workload):
    from gamedev_b200 import GD_SEARCH_MORTON, workloads

    cfg = workloads.config(workload)
    wedge, width, idm = gd.wedge_info(cfg)
    f = np.float32
    x_min, x_max = f(cfg.x_min), f(cfg.x_max)
    # X_WEDGE (const_defs.cuh:56-57)
    assert wedge == bool(cfg.n_x > 1 and x_max - x_min < f(6.28318530717958647692) - f(1.0e-06))
    assert wedge == workload.startswith("w")
    if not wedge:
        assert width == 0.0 and idm == -1.0
        return
    # the image rotation angle of each search (col_site_init.cu:60, morton_ghost.cuh:62)
    want = (x_max - x_min) if cfg.search == GD_SEARCH_MORTON else f(cfg.x_max - cfg.x_min)
    assert f(width) == want
    # _get_image_dist_min (param_grid.cuh:86-89) with the host's sinf
    sinf = _libm_sinf()
    y_min, z_min, z_max = f(cfg.y_min), f(cfg.z_min), f(cfg.z_max)
    expect = f(2.0) * y_min * min(sinf(z_min), sinf(z_max)) * abs(sinf(f(0.5) * (x_max - x_min)))
    assert f(idm).view(np.uint32) == f(expect).view(np.uint32)


@pytest.mark.parametrize("workload", ["w0_wedge_3d", "w1_narrow_2d", "w2_wide_3d"])
def test_wedge_swarms_lie_inside_the_wedge(workload):
    from gamedev_b200 import workloads

    cfg = workloads.config(workload)
    p = workloads.particles(workload, n=4096)
    assert (p[:, 0] >= cfg.x_min).all() and (p[:, 0] < cfg.x_max).all()
    assert cfg.n_x > 1 and cfg.x_max - cfg.x_min < 2.0 * math.pi


def test_morton_ghost_rule_cases():
    """The oracle's ghost rule (morton_gcount, morton_ghost.cuh:28-50) on hand-placed sites of a
    3.8 rad wedge [0, 3.8): image 2 (+width) stands for the x_min seam and is kept within q_max of
    it, image 1 (-width) for the x_max seam; past a quarter turn from a seam the distance is the
    cylindrical radius, not the plane distance."""
    from oracle import oracle

    x_min, x_max, q_max = 0.0, 3.8, 0.5
    R = np.array([1.0, 1.0, 1.0, 10.0, 0.4, 1.0], np.float64)
    th = np.array([0.1, 3.75, 1.9, 0.01, 1.9, 3.8 - 2.0], np.float64)
    site4 = np.zeros((R.size, 4), np.float32)
    site4[:, 0] = R * np.cos(th)
    site4[:, 1] = R * np.sin(th)
    keep, margin = oracle.morton_ghosts(site4, th.astype(np.float32), q_max, x_min, x_max)
    want = np.array([
        [False, True],   # 0.1 rad past x_min: sin(0.1) = 0.0998 <= 0.5; 3.7 rad before x_max (cos < 0): R
        [True, False],   # 0.05 rad before x_max
        [False, False],  # the middle: 1.9 rad from both seams, beyond a quarter turn, R = 1 > 0.5
        [False, True],   # R = 10: 10 sin(0.01) = 0.1 <= 0.5
        [True, True],    # R = 0.4 <= q_max: both seams within reach whatever the angle
        [False, False],  # 2.0 rad from x_max (cos < 0, so R = 1) and 1.8 rad from x_min (R)
    ])
    assert np.array_equal(keep, want), keep
    assert np.all(np.abs(margin) > 1e-3)


def _morton_ghost_rows(all_codes, all_d2, k, unique_ids):
    """_morton_ghost_topk's selection (morton/morton_query.cuh:62-140) from an owner's ascending
    candidate list: without unique ids, the 3K nearest records, sorted by (particle, d^2, code),
    the first of each particle kept, then the K nearest of those; with unique ids, the K nearest."""
    rows = []
    for codes, d2 in zip(all_codes, all_d2):
        keep = codes >= 0
        cand = list(zip(d2[keep].view(np.uint32).tolist(), codes[keep].tolist()))  # ascending keys
        if not unique_ids:
            cand = sorted(cand[:3 * k], key=lambda t: (t[1] // 3, t[0], t[1]))
            cand = [t for j, t in enumerate(cand) if j == 0 or t[1] // 3 != cand[j - 1][1] // 3]
            cand.sort()
        row = [c for _, c in cand[:k]]
        rows.append(row + [-1] * (k - len(row)))
    return np.array(rows, np.int32)


def test_morton_ghost_selection_equals_the_heap_dedup():
    """The Morton search keeps only the 3K nearest records before removing duplicate images.  That
    loses nothing: the K nearest particles by their nearest image lie among the 3K - 2 nearest
    records, since each particle has at most three.  So its rows equal the KD heap's in-place dedup
    (gdo_knn_brute_images), for every K, with the decision taken from the largest q."""
    from oracle import oracle

    n, width = 200, 0.05
    sites = _wedge_sites(n, width, seed=23)
    rng = np.random.default_rng(5)
    q = rng.uniform(0.05, 0.5, n).astype(np.float32)
    active = np.ones(n, np.uint8)
    active[::13] = 0
    act = active.astype(bool)
    all_codes, all_d2 = oracle.knn_brute_images(sites, n, q, active, 3 * n, -1.0)
    all_codes, all_d2 = all_codes[act], all_d2[act]
    for k in (1, 5, 17, 40):
        for idm in (0.1, 2.0):  # dedup on (image_dist_min <= 2 q_max) and off
            unique = not (idm <= 2.0 * float(q.max()))
            want = _morton_ghost_rows(all_codes, all_d2, k, unique)
            got, _ = oracle.knn_brute_images(sites, n, q, active, k, idm, q_dedup=float(q.max()))
            assert np.array_equal(got[act], want), (k, idm)
