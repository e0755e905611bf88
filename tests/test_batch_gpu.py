"""Batched neighbour search (gd_batch_*): many swarms of uneven size and K in one persistent
top-K launch.  Bar: every swarm's codes, measure and K-th d^2 bit-identical to the one-swarm path
(gd_geometry_build + gd_knn) on that swarm alone; the same after a CUDA graph capture and replay;
a non-finite particle in one swarm reported by gd_batch_check with its concatenated index."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solo(gd, cfg, p, k):
    import torch

    cfg.n_k = k
    sw = gd.SwarmCollision(cfg, len(p))
    codes, measure, kth = sw.knn(gd.particles_to_device(p))
    torch.cuda.synchronize()
    out = codes.cpu().numpy(), measure.cpu().numpy(), kth.cpu().numpy()
    sw.close()
    return out


def _compare(batch, codes, measure, kth, solos):
    c = codes.cpu()
    m = measure.cpu()
    t = kth.cpu()
    for s, (sc, sm, st) in enumerate(solos):
        assert np.array_equal(batch.codes_of(c, s).numpy(), sc), s
        assert np.array_equal(batch.rows_of(m, s).numpy().view(np.uint64), sm.view(np.uint64)), s
        assert np.array_equal(batch.rows_of(t, s).numpy().view(np.uint32), st.view(np.uint32)), s


def test_batch_matches_solo_runs_and_graph_replay(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    cfg, sizes, ks, p = workloads.c2_batch(swarms=12, seed=7, n_min=100, n_max=40000)
    batch = gd.SwarmBatch(cfg, sizes, ks)
    dp = gd.particles_to_device(p)
    off = batch.part_off
    solos = [_solo(gd, workloads.c2_batch(swarms=12, seed=7, n_min=100, n_max=40000)[0],
                   p[off[s]:off[s + 1]], ks[s]) for s in range(len(sizes))]
    codes, measure, kth = batch.outputs()
    for _ in range(2):  # two calls in a row: nothing carries over
        codes.fill_(-7)
        batch.knn(dp, codes, measure, kth)
        batch.check()
        torch.cuda.synchronize()
        _compare(batch, codes, measure, kth, solos)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        batch.knn(dp, codes, measure, kth)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batch.knn(dp, codes, measure, kth)
    codes.fill_(-7)
    graph.replay()
    batch.check()
    torch.cuda.synchronize()
    _compare(batch, codes, measure, kth, solos)

    bad = int(off[5]) + 17
    dp[bad, 2] = float("inf")
    graph.replay()
    with pytest.raises(gd.GdError) as e:
        batch.check()
    assert e.value.status == 3 and e.value.detail == bad
    del graph
    batch.close()
