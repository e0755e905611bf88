"""The radius-bounded range query (gd_range.cu: a warp per owner, candidates inside min(q, r)
collected by ballot and sorted by a warp-wide bitonic network; the owners it cannot serve go to the
per-lane heap query with the full q).

Bar: for every proposal below, the rows, the FP64 measures and the K-th d^2 equal the plain query's
bit for bit, with the range query on and off.  Proposals cover the cases the kernel branches on:
  * near the true K-th distance (the common case: a little more than K sites inside);
  * exactly the K-th distance (float rounding of r*r can leave K - 1 inside: a fallback);
  * shorter (fewer than K inside: the whole q ball is searched, or the heap query takes the owner
    when that ball is too large) and much longer (more than the 128 candidates an owner may hold: the
    K-th nearest of the first 128 bounds a rescan);
  * r >= q, r = 0, r = inf, NaN and negative r (the bound falls back to q, or to nothing);
on 3D, 2D and radial-only shapes, odd and small K, and a swarm of a single bucket.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(gd, workload, n, K, seed=5):
    import torch

    from gamedev_b200 import workloads

    cfg = workloads.config(workload)
    cfg.n_k = K
    p = workloads.particles(workload, n=n, seed=seed)
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p)
    codes, measure, kth = sw.knn(dp)
    torch.cuda.synchronize()
    return cfg, sw, dp, codes, measure, kth


def _bounded(sw, dp, radius, codes, range_query):
    import torch

    sw.set_tuning(range_query=range_query)
    c = torch.empty_like(codes)
    m = torch.empty((codes.shape[0],), dtype=torch.float64, device=codes.device)
    k = torch.empty((codes.shape[0],), dtype=torch.float32, device=codes.device)
    st = torch.zeros(4, dtype=torch.int64, device=codes.device)
    sw.col_cache_get_bounded(dp, radius, c, m, k, st)
    torch.cuda.synchronize()
    return c, m, k, st


def _proposals(kth, q, gen):
    import torch

    n = kth.shape[0]
    r0 = kth.double().sqrt()
    u = torch.rand(n, device="cuda", generator=gen, dtype=torch.float64)
    kind = torch.randint(0, 10, (n,), device="cuda", generator=gen)
    r = torch.empty(n, dtype=torch.float64, device="cuda")
    r = torch.where(kind == 0, r0 * (1.0 + 0.05 * u), r)        # near: the common case
    r = torch.where(kind == 1, r0, r)                             # exactly the K-th distance
    r = torch.where(kind == 2, r0 * (0.5 + 0.49 * u), r)          # short: fallbacks
    r = torch.where(kind == 3, r0 * (2.0 + 2.0 * u), r)           # long: too many candidates
    r = torch.where(kind == 4, q.double() * (1.0 + u), r)         # at or beyond q
    r = torch.where(kind == 5, torch.zeros_like(r), r)            # nothing inside but the owner
    r = torch.where(kind == 6, torch.full_like(r, math.inf), r)
    r = torch.where(kind == 7, torch.full_like(r, math.nan), r)
    r = torch.where(kind == 8, r0 * (1.0 + 0.005 * u), r)         # very tight
    r = torch.where(kind == 9, -q.double() * (2.0 + u), r)        # negative: bounds nothing
    return r.float()


@pytest.mark.parametrize("workload,n,K", [("c3_learned_3d", 1 << 17, 64), ("c3_learned_3d", 1 << 16, 33),
                                          ("c3_learned_3d", 1 << 16, 7), ("c3_learned_3d", 1 << 16, 1),
                                          ("c1_multisize_2d", 1 << 16, 64), ("v0_radial_units", 4096, 16),
                                          ("c0_plain_small", 20, 8)])
def test_range_query_equals_plain_rows(gd, cuda, workload, n, K):
    import torch

    cfg, sw, dp, codes, measure, kth = _setup(gd, workload, n, K)
    site4, q, active = sw.get_sites()
    gen = torch.Generator(device="cuda").manual_seed(n + K)
    radius = _proposals(kth, q, gen)
    for rq in (1, 0):
        c, m, k, st = _bounded(sw, dp, radius, codes, rq)
        assert torch.equal(codes, c), (workload, K, rq, int((codes != c).any(dim=1).sum().item()))
        assert torch.equal(measure.view(torch.int64), m.view(torch.int64)), (workload, K, rq)
        assert torch.equal(kth.view(torch.int32), k.view(torch.int32)), (workload, K, rq)
    sw.close()


def test_range_query_serves_good_proposals_without_fallback(gd, cuda):
    """With proposals a few per cent above the true K-th distance every owner is served by the range
    query itself: no fallback, and about K candidates collected per owner.  (At 2^20 owners every
    q-ball of the c3 disk holds more than K sites, so no row is short.)"""
    import torch

    n, K = 1 << 20, 64
    cfg, sw, dp, codes, measure, kth = _setup(gd, "c3_learned_3d", n, K)
    site4, q, active = sw.get_sites()
    radius = (kth.double().sqrt() * 1.02).float()
    c, m, k, st = _bounded(sw, dp, radius, codes, 1)
    assert torch.equal(codes, c) and torch.equal(kth.view(torch.int32), k.view(torch.int32))
    n_act = int(active.sum().item())
    # owners whose row is not full even at q (a handful at the disk edges) still need the full walk
    incomplete = int(((codes < 0).any(dim=1) & (active > 0)).sum().item())
    assert int(st[3].item()) <= incomplete + n_act // 1000, (int(st[3].item()), incomplete)
    cand = int(st[2].item()) / n_act
    assert K <= cand < 1.3 * K, cand
    sw.close()


def test_range_query_hands_large_balls_to_the_heap_query(gd, cuda):
    """A search radius q four times the default makes every q ball hold thousands of sites: owners
    with short proposals then outgrow the range query's lists and go to the per-lane heap query.
    Rows stay identical to the plain query's."""
    import torch

    from gamedev_b200 import workloads

    n, K = 1 << 18, 64
    cfg = workloads.config("c3_learned_3d")
    cfg.h_search = 4.0
    p = workloads.particles("c3_learned_3d", n=n, seed=9)
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p)
    codes, measure, kth = sw.knn(dp)
    gen = torch.Generator(device="cuda").manual_seed(2)
    u = torch.rand(n, device="cuda", generator=gen, dtype=torch.float64)
    radius = (kth.double().sqrt() * torch.where(u < 0.5, 0.3 + 0.5 * u, 1.0 + 0.02 * u)).float()
    c, m, k, st = _bounded(sw, dp, radius, codes, 1)
    assert torch.equal(codes, c)
    assert torch.equal(measure.view(torch.int64), m.view(torch.int64))
    assert torch.equal(kth.view(torch.int32), k.view(torch.int32))
    assert int(st[3].item()) > 0
    sw.close()
