"""The collision operator inside a caller's CUDA graph.

gd_collision_operator enqueues the bath-start pass and a conditional WHILE node whose body is one
wave; every decision of the reference's host controller loop (_col_chain.cuh:215-537) runs on the
device, so a caller can capture operators into its own graph.  Bars:
  * two operators captured in one graph and replayed twice give the particles, the RNG streams and
    the summed statistics of four eager operators bit for bit, and their bath records under the
    reference validator's repeat comparison (the audit sums are FP64 atomics, whose order varies
    from run to run in the reference too: equal to 1e-12, decisions and counts exactly);
  * an error met inside a replay (a non-finite grain count the controller rejects) is returned by
    gd_check_operator after the replay, and the handle runs clean input afterwards.
"""

import math

import numpy as np
import pytest

from tests.test_collide_gpu import _controller_equivalent

pytestmark = pytest.mark.gpu


def _mass(p):
    return float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())


def _setup(gd, cfg, p, seed):
    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    sw.build_cache(dp)
    rng = gd.rngstate_init(len(p), seed=seed)
    return sw, dp, rng


def _duration(gd, cfg, p, mass):
    from gamedev_b200 import workloads

    sw, dp, rng = _setup(gd, cfg, p, 5)
    sw.evolve_local_collisions(dp, rng, 1.0e-9 * workloads.orbital_time(), mass)
    rate_max = float(sw.owner_state()[0][:, 0].max().item())
    sw.close()
    # ~20 expected events for the fastest owner: the change bounds split it into many waves
    return 20.0 / rate_max


def test_captured_operators_equal_eager(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    cfg = workloads.config("c1_multisize_2d")
    p = workloads.particles("c1_multisize_2d", n=20000)
    mass = _mass(p)
    dur = _duration(gd, cfg, p, mass)

    sw, dp, rng = _setup(gd, cfg, p, 7)
    eager = []
    for _ in range(4):
        sw.evolve_local_collisions(dp, rng, dur, mass)
        eager.append(sw.last_operator_stats())
    torch.cuda.synchronize()
    e_part = dp.cpu().numpy()
    e_uni = gd.rng_uniforms(rng, len(p), 4).cpu().numpy()
    e_sum = sw.controller_summary()
    sw.close()

    sw, dp, rng = _setup(gd, cfg, p, 7)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sw.evolve_local_collisions(dp, rng, dur, mass)
        sw.evolve_local_collisions(dp, rng, dur, mass)
    captured = []
    for _ in range(2):
        graph.replay()
        sw.check_operator()
        captured.append(sw.last_operator_stats())
    torch.cuda.synchronize()
    c_part = dp.cpu().numpy()
    c_uni = gd.rng_uniforms(rng, len(p), 4).cpu().numpy()
    c_sum = sw.controller_summary()

    assert np.array_equal(e_part.view(np.uint64), c_part.view(np.uint64))
    assert np.array_equal(e_uni, c_uni)
    for k in range(2):
        a, b, c = eager[2 * k], eager[2 * k + 1], captured[k]
        assert c["waves"] == a["waves"] + b["waves"] and c["chain_launches"] == c["waves"]
        assert c["owner_updates"] == a["owner_updates"] + b["owner_updates"]
        assert c["events"] == a["events"] + b["events"]
        assert c["min_duration"] == min(a["min_duration"], b["min_duration"])
        assert c["max_duration"] == max(a["max_duration"], b["max_duration"])
    assert min(s["waves"] for s in eager) >= 2  # the wave body runs more than once per operator
    assert _controller_equivalent(e_sum, c_sum)
    assert c_sum["operator_count"] == 4 and c_sum["bath_count"] > 4
    flags = ("activity_overshoot", "distribution_overshoot", "persistent_overshoot", "group", "bath")
    assert [[r[f] for f in flags] for r in e_sum["baths"]] == [[r[f] for f in flags] for r in c_sum["baths"]]

    # an error inside a replay is the status of the next check; clean input runs afterwards
    saved = dp[321].clone()
    dp[321, 7] = float("nan")
    graph.replay()
    with pytest.raises(gd.GdError) as e:
        sw.check_operator()
    assert e.value.status in (4, 8)
    dp[321] = saved
    sw.evolve_local_collisions(dp, rng, dur, mass)
    graph.replay()
    sw.check_operator()
    torch.cuda.synchronize()
    assert np.isfinite(dp.cpu().numpy()).all()
    del graph
    sw.close()
