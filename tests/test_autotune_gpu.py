"""Speed-only settings of the neighbour search and the autotuner (gd_set_tuning, gd_autotune,
gd_batch_set_tuning).  Bar: every setting (sort order, walk, prescan depth, block width) gives
codes, measure and K-th d^2 bit-identical to the default setting, plain and radius-bounded; the
autotuner returns a valid setting, leaves it in the handle and its lists are exact."""

import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(sw, dp, radius=None):
    import torch

    n, K = sw.n_p, sw.n_k
    c = torch.empty((n, K), dtype=torch.int32, device="cuda")
    m = torch.empty(n, dtype=torch.float64, device="cuda")
    k = torch.empty(n, dtype=torch.float32, device="cuda")
    sw.col_site_init(dp)
    if radius is None:
        sw.col_cache_get(dp, c, m, k)
    else:
        sw.col_cache_get_bounded(dp, radius, c, m, k, None)
    torch.cuda.synchronize()
    return c, m, k


def _same(a, b):
    import torch

    return (torch.equal(a[0], b[0]) and torch.equal(a[1].view(torch.int64), b[1].view(torch.int64))
            and torch.equal(a[2].view(torch.int32), b[2].view(torch.int32)))


@pytest.mark.parametrize("workload", ["c3_learned_3d", "c1_multisize_2d"])
def test_every_setting_gives_the_same_lists(gd, cuda, workload):
    from gamedev_b200 import workloads

    cfg = workloads.config(workload)
    p = workloads.particles(workload, n=1 << 17, seed=41)
    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    ref = _run(sw, dp)
    radius = (ref[2].double().sqrt() * 1.07).float()
    ref_b = _run(sw, dp, radius)
    assert _same(ref, ref_b)
    dim = 3 if cfg.n_z > 1 else 2
    for bfs, pre, w, sb in itertools.product((0, 1), (0, 1, 3), (1, 4), (0, 16 * dim)):
        sw.set_tuning(walk_breadth_first=bfs, prescan=pre, warps_per_block=w, sort_bits=sb)
        assert _same(_run(sw, dp), ref), (bfs, pre, w, sb)
        assert _same(_run(sw, dp, radius), ref), (bfs, pre, w, sb)
    sw.close()


def test_autotune_keeps_exact_lists(gd, cuda):
    from gamedev_b200 import workloads

    cfg = workloads.config("c3_learned_3d")
    p = workloads.particles("c3_learned_3d", n=1 << 18, seed=42)
    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    ref = _run(sw, dp)
    best, ms = sw.autotune(dp)
    assert ms > 0 and best == sw.tuning()
    assert best["sort_bits"] in (0, 48) and best["prescan"] in (1, 2, 3) and best["walk_breadth_first"] in (0, 1)
    assert _same(_run(sw, dp), ref)
    radius = (ref[2].double().sqrt() * 1.07).float()
    best_b, _ = sw.autotune(dp, radius, tune_sort=False)
    assert best_b["sort_bits"] == best["sort_bits"]
    assert _same(_run(sw, dp, radius), ref)
    with pytest.raises(gd.GdError):
        sw.set_tuning(sort_bits=12)  # fewer than 16 bits per axis
    sw.close()


def test_batch_tuning_keeps_solo_lists(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    cfg, sizes, ks, p = workloads.c2_batch(swarms=6, seed=9, n_min=200, n_max=20000)
    dp = gd.particles_to_device(p)
    batch = gd.SwarmBatch(cfg, sizes, ks)
    codes, measure, kth = batch.outputs()
    batch.knn(dp, codes, measure, kth)
    batch.check()
    ref = (codes.clone(), measure.clone(), kth.clone())
    batch.set_tuning(warps_per_block=2, prescan=1, walk_breadth_first=0, sort_bits=48)
    batch.knn(dp, codes, measure, kth)
    batch.check()
    torch.cuda.synchronize()
    assert _same((codes, measure, kth), ref)
    batch.close()
