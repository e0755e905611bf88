"""The learned neighbour-search step captured in one CUDA graph.

With the non-finite screen deferred (gd_set_deferred_checks), geometry build, radius features,
MLP radius proposal and radius-bounded top-K enqueue without a host synchronisation, so the step is
captured once and replayed on new particle positions written into the same buffer.  Bar: every
replay's codes, measure and K-th d^2 bit-identical to the eager plain query on the same positions;
a non-finite particle written into the buffer is reported by gd_check_geometry after the replay,
with its index, and the next clean replay is exact again.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_step_graph_replays_are_exact(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    n = 1 << 17
    cfg = workloads.config("c3_learned_3d")
    p = workloads.particles("c3_learned_3d", n=n, seed=31)
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    sw = gd.SwarmCollision(cfg, n)
    ref = gd.SwarmCollision(cfg, n)  # eager plain query, the judge of every replay
    dp = gd.particles_to_device(p)
    K = cfg.n_k
    codes0, measure0, kth0 = sw.knn(dp)
    model = gd.RadiusModel(cfg.R_0, seed=3)
    feats = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    prev = kth0.clone()
    dt = 0.02 * workloads.orbital_time()
    for _ in range(3):  # a few drifted plain steps train the network
        sw.drift_keplerian(dp, dt)
        sw.col_site_init(dp)
        sw.col_cache_get(dp, codes0, measure0, kth0)
        sw.radius_features(dp, prev, mass, out=feats)
        model.train(feats, kth0, iterations=60, batch=16384, lr=2e-3)
        prev.copy_(kth0)
    model.calibrate(feats, kth0, 0.999)

    sw.set_deferred_checks(True)
    radius = torch.empty(n, dtype=torch.float32, device="cuda")
    codes = torch.empty((n, K), dtype=torch.int32, device="cuda")
    measure = torch.empty(n, dtype=torch.float64, device="cuda")
    kth = torch.empty(n, dtype=torch.float32, device="cuda")

    def step():
        sw.col_site_init(dp)
        sw.radius_features(dp, prev, mass, out=feats)
        model.predict(feats, out=radius)
        sw.col_cache_get_bounded(dp, radius, codes, measure, kth, None)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        step()  # warm-up outside capture (sets kernel attributes once)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()

    rc = torch.empty_like(codes)
    rm = torch.empty_like(measure)
    rk = torch.empty_like(kth)
    for it in range(3):
        sw.drift_keplerian(dp, dt)  # new positions in the captured buffer
        graph.replay()
        sw.check_geometry()
        ref.col_site_init(dp)
        ref.col_cache_get(dp, rc, rm, rk)
        torch.cuda.synchronize()
        assert torch.equal(codes, rc), it
        assert torch.equal(measure.view(torch.int64), rm.view(torch.int64)), it
        assert torch.equal(kth.view(torch.int32), rk.view(torch.int32)), it
        prev.copy_(kth)

    # a non-finite particle: the replay runs past it, the deferred check reports it
    saved = dp[777].clone()
    dp[777, 1] = float("nan")
    graph.replay()
    with pytest.raises(gd.GdError) as e:
        sw.check_geometry()
    assert e.value.status == 3 and e.value.detail == 777
    dp[777] = saved
    graph.replay()
    sw.check_geometry()
    ref.col_site_init(dp)
    ref.col_cache_get(dp, rc, rm, rk)
    torch.cuda.synchronize()
    assert torch.equal(codes, rc)
    del graph
    model.close()
    sw.close()
    ref.close()
