"""The CPU oracle's exact top-K, checked against itself (KD tree vs brute force) and against the
invariants the reference's KNN suite asserts (val/swarm/mod/test_knn/knn_benchmark.cu:322-420,
508-548): identical identifiers, rows sorted by (d^2, identifier), d^2 within the search radius,
inactive sites never returned."""

import math

import numpy as np
import pytest

from tests import cases


@pytest.fixture(scope="module")
def all_cases(gd):
    return cases.small_cases(gd)


def _row_invariants(codes, d2, q, active):
    n, k = codes.shape
    for i in range(n):
        row, dr = codes[i], d2[i]
        if not active[i]:
            assert (row == -1).all()
            continue
        valid = row >= 0
        nv = int(valid.sum())
        assert valid[:nv].all() and not valid[nv:].any(), "padding must trail"
        keys = [(float(dr[s]), int(row[s])) for s in range(nv)]
        assert keys == sorted(keys)
        assert len(set(row[:nv].tolist())) == nv
        assert (dr[:nv] <= np.float32(q[i]) * np.float32(q[i])).all()
        assert all(active[c // 3] for c in row[:nv])
        assert (row[:nv] % 3 == 0).all()  # full disk: physical images only


@pytest.mark.parametrize("idx", range(11))
def test_kdtree_equals_brute_force(oracle_lib, all_cases, idx):
    name, cfg, p = all_cases[idx]
    site4, q, active, bad = oracle_lib.site_init(cfg, p)
    assert bad == -1
    cb, db = oracle_lib.knn_brute(site4, q, active, cfg.n_k)
    ck, dk = oracle_lib.knn_kdtree(site4, q, active, cfg.n_k)
    assert np.array_equal(cb, ck), name
    assert np.array_equal(db.view(np.uint32), dk.view(np.uint32)), name
    _row_invariants(ck, dk, q, active)


def test_self_is_first_neighbour(oracle_lib, all_cases):
    name, cfg, p = all_cases[0]
    site4, q, active, _ = oracle_lib.site_init(cfg, p)
    codes, d2 = oracle_lib.knn_kdtree(site4, q, active, cfg.n_k)
    idx = np.arange(len(p))
    act = active.astype(bool)
    # no coincident sites in this case: the owner itself is the unique d^2 = 0 neighbour
    assert (codes[act, 0] == 3 * idx[act]).all()
    assert (d2[act, 0] == 0).all()


def test_coincident_sites_tie_break_by_code(oracle_lib, all_cases):
    name, cfg, p = [c for c in all_cases if c[0] == "coincident_k24"][0]
    site4, q, active, _ = oracle_lib.site_init(cfg, p)
    codes, d2 = oracle_lib.knn_kdtree(site4, q, active, cfg.n_k)
    zero = d2 == 0
    # among d^2 == 0 entries, codes ascend and the owner is among them
    for i in range(len(p)):
        z = codes[i][zero[i] & (codes[i] >= 0)]
        assert (np.diff(z) > 0).all()
        assert 3 * i in z


def test_radius_bound_pads_with_minus_one(oracle_lib, all_cases):
    name, cfg, p = [c for c in all_cases if c[0] == "radius_bound_fewer_than_k"][0]
    site4, q, active, _ = oracle_lib.site_init(cfg, p)
    codes, d2 = oracle_lib.knn_kdtree(site4, q, active, cfg.n_k)
    counts = (codes >= 0).sum(axis=1)
    assert counts.min() >= 1 and counts.max() < cfg.n_k  # every row truncated by the radius


def test_inactive_sites_are_filtered(oracle_lib, all_cases):
    name, cfg, p = [c for c in all_cases if c[0] == "inactive_filter"][0]
    site4, q, active, _ = oracle_lib.site_init(cfg, p)
    assert 0 < active.sum() < len(p)
    codes, _ = oracle_lib.knn_kdtree(site4, q, active, cfg.n_k)
    inact = np.nonzero(active == 0)[0]
    assert (codes[inact] == -1).all()
    assert not np.isin(codes[codes >= 0] // 3, inact).any()


def test_nonfinite_particle_reported(oracle_lib, gd):
    cfg = cases.code_unit_config(gd)
    p = cases.random_swarm(cfg, 100, 3)
    p[57, 4] = np.nan
    p[80, 7] = np.inf
    _, _, active, bad = oracle_lib.site_init(cfg, p)
    assert bad == 57 and active[57] == 0 and active[80] == 0


def test_measure_of_full_ball_inside_domain(oracle_lib, gd):
    # _get_ball_measure: a 3D ball away from every bound is 4/3 pi r^3
    cfg = cases.code_unit_config(gd)
    p = np.zeros((1, 8))
    p[0, 1], p[0, 2] = 1.0, 0.5 * math.pi
    m = oracle_lib.ball_measure(cfg, p, np.ones(1, np.uint8), np.array([0.01 ** 2], np.float32))
    r = math.sqrt(float(np.float32(0.01 ** 2)))
    assert m[0] == pytest.approx(4.0 * math.pi * r ** 3 / 3.0, rel=1e-15)


def test_reference_heap_rows_sort_to_canonical_order(oracle_lib, all_cases):
    """oracle.ref.refknn.canonical turns a heap-ordered reference cache (any row permutation, empty
    slots carrying d^2 = q^2) into the ascending (d^2, code) rows the B200 search writes."""
    from oracle.ref import refknn

    name, cfg, p = all_cases[6]  # radius-bounded: rows with fewer than K neighbours
    site4, q, active, _ = oracle_lib.site_init(cfg, p)
    codes, d2 = oracle_lib.knn_brute(site4, q, active, cfg.n_k)
    rng = np.random.default_rng(5)
    perm = np.argsort(rng.random(codes.shape), axis=1)
    hc = np.take_along_axis(codes, perm, axis=1)
    hd = np.take_along_axis(np.where(codes >= 0, d2, (q * q)[:, None]).astype(np.float32), perm, axis=1)
    c, _, kth = refknn.canonical(hc, hd)
    assert (codes < 0).any(), name
    assert np.array_equal(c, codes)
    assert np.array_equal(kth.view(np.uint32), oracle_lib.kth_from_rows(codes, d2).view(np.uint32))
