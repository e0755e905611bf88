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


def test_batched_operators_equal_solo_operators(gd, cuda):
    """gd_batch_collide: every swarm's collision operator on the batch's rows, side by side (eager,
    and captured with the batch search into one graph and replayed), gives each swarm the
    particles and RNG streams of gd_collision_operator on that swarm alone, bit for bit; an
    operator error names its swarm."""
    import math

    import torch

    from gamedev_b200 import workloads

    S = 12
    cfg, sizes, ks, p = workloads.c2_batch(swarms=S, seed=9, n_min=500, n_max=30000)
    off = [int(v) for v in np.concatenate([[0], np.cumsum(sizes)])]
    masses = [float((p[off[s]:off[s + 1], 7] * math.pi * p[off[s]:off[s + 1], 6] ** 3 / 6.0).sum())
              for s in range(S)]
    # ~10 expected events for each swarm's fastest owner (bath-start rate of a short operator)
    durations = []
    for s in range(S):
        c = workloads.c2_batch(swarms=S, seed=9, n_min=500, n_max=30000)[0]
        c.n_k = ks[s]
        sw = gd.SwarmCollision(c, sizes[s])
        dps = gd.particles_to_device(p[off[s]:off[s + 1]])
        sw.evolve_collisions(dps, gd.rngstate_init(sizes[s], seed=3), 1.0e-12 * workloads.orbital_time(), masses[s])
        durations.append(10.0 / float(sw.owner_state()[0][:, 0].max().item()))
        sw.close()

    def solo(s, operators):
        c = workloads.c2_batch(swarms=S, seed=9, n_min=500, n_max=30000)[0]
        c.n_k = ks[s]
        sw = gd.SwarmCollision(c, sizes[s])
        dps = gd.particles_to_device(p[off[s]:off[s + 1]])
        rng = gd.rngstate_init(sizes[s], seed=11 + s)
        for _ in range(operators):
            sw.evolve_collisions(dps, rng, durations[s], masses[s])
        torch.cuda.synchronize()
        out = dps.cpu().numpy(), gd.rng_uniforms(rng, sizes[s], 3).cpu().numpy(), sw.last_operator_stats()
        sw.close()
        return out

    def batch_rng():
        return torch.cat([gd.rngstate_init(sizes[s], seed=11 + s) for s in range(S)])

    batch = gd.SwarmBatch(cfg, sizes, ks)
    codes, measure, kth = batch.outputs()
    dp = gd.particles_to_device(p)
    rng = batch_rng()
    batch.knn(dp, codes, measure, kth)
    batch.check()
    batch.collide(dp, rng, codes, measure, durations, masses)
    torch.cuda.synchronize()
    got = dp.cpu().numpy()
    for s in range(S):
        ref_p, ref_u, ref_st = solo(s, 1)
        assert np.array_equal(got[off[s]:off[s + 1]].view(np.uint64), ref_p.view(np.uint64)), s
        u = gd.rng_uniforms(rng.view(-1, gd.rng_state_bytes())[off[s]:off[s + 1]], sizes[s], 3).cpu().numpy()
        assert np.array_equal(u, ref_u), s
        st = batch.operator_stats(s)
        assert st["waves"] == ref_st["waves"] and st["events"] == ref_st["events"], s

    # the search and the operators of all swarms captured into one graph and replayed twice: the
    # particles of two solo operators per swarm
    dp.copy_(gd.particles_to_device(p))
    rng.copy_(batch_rng())
    batch.reset_controller()  # the solo runs start with fresh bath controllers too
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        batch.knn(dp, codes, measure, kth)
        batch.collide(dp, rng, codes, measure, durations, masses)
    for _ in range(2):
        graph.replay()
        batch.check()
    torch.cuda.synchronize()
    got = dp.cpu().numpy()
    for s in range(S):
        ref_p, ref_u, _ = solo(s, 2)
        assert np.array_equal(got[off[s]:off[s + 1]].view(np.uint64), ref_p.view(np.uint64)), s

    # a non-finite grain count in swarm 4: the screen names the particle, the operator its swarm
    bad = off[4] + 5
    dp[bad, 7] = float("nan")
    with pytest.raises(gd.GdError) as e:
        batch.collide(dp, rng, codes, measure, durations, masses)
    assert e.value.status in (4, 8) and e.value.detail == 4
    del graph
    batch.close()


def test_batch_at_the_full_batched_shape(gd, cuda):
    """The batched configuration itself: 256 swarms of 2^10 to 2^18 particles (about 1.2e7 in all),
    K from {16, 32, 64}, one persistent search.  Every swarm's rows, measures and K-th d^2 equal a
    solo search of that swarm."""
    import torch

    from gamedev_b200 import workloads

    cfg, sizes, ks, p = workloads.c2_batch()
    assert len(sizes) == 256 and min(sizes) >= 1 << 10 and max(sizes) <= 1 << 18
    batch = gd.SwarmBatch(cfg, sizes, ks)
    dp = gd.particles_to_device(p)
    codes, measure, kth = batch.outputs()
    batch.knn(dp, codes, measure, kth)
    batch.check()
    torch.cuda.synchronize()
    c, m, t = codes.cpu(), measure.cpu(), kth.cpu()
    del codes, measure, kth, dp
    off = batch.part_off
    for s in range(len(sizes)):
        sc, sm, st = _solo(gd, workloads.c2_batch()[0], p[off[s]:off[s + 1]], ks[s])
        assert np.array_equal(batch.codes_of(c, s).numpy(), sc), s
        assert np.array_equal(batch.rows_of(m, s).numpy().view(np.uint64), sm.view(np.uint64)), s
        assert np.array_equal(batch.rows_of(t, s).numpy().view(np.uint32), st.view(np.uint32)), s
    batch.close()
