"""gd_knn_static, the neighbour search that allocates no device memory (for callers that may not
call cudaMalloc while they run), against the handle-based entry point (gd_create +
gd_geometry_build + gd_knn) on the same particles.

Bar: codes, measure and K-th d^2 bit-identical to the handle path on consecutive calls with
different swarms (3D at the 65536-particle maximum, a ragged 2D swarm, then both again), so nothing
left in the shared scratch by one call leaks into the next; device free memory unchanged across
warm calls; an oversize swarm rejected before any device work; a non-finite particle reported with
its index and the scratch usable again afterwards.

This file is named to be collected last, so that it also runs after every other GPU test in one
process.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(gd):
    from gamedev_b200 import workloads

    cfg_a = workloads.config("c0_plain_small")
    p_a = workloads.particles("c0_plain_small", n=gd.STATIC_MAX_PARTICLES, seed=21)
    cfg_b = workloads.config("c1_multisize_2d")
    p_b = workloads.particles("c1_multisize_2d", n=50001, seed=22)
    return (cfg_a, p_a), (cfg_b, p_b)


def _handle_knn(gd, cfg, dp):
    import torch

    sw = gd.SwarmCollision(cfg, int(dp.shape[0]))
    codes, measure, kth = sw.knn(dp)
    torch.cuda.synchronize()
    out = codes.cpu().numpy(), measure.cpu().numpy(), kth.cpu().numpy()
    sw.close()
    return out


def _outputs(cfg, n):
    import torch

    # sentinels, so that every element the call must write is seen to be written
    return (torch.full((n, cfg.n_k), -7, dtype=torch.int32, device="cuda"),
            torch.full((n,), -7.0, dtype=torch.float64, device="cuda"),
            torch.full((n,), -7.0, dtype=torch.float32, device="cuda"))


def _assert_same(got, want, name):
    codes, measure, kth = (t.cpu().numpy() for t in got)
    assert np.array_equal(codes, want[0]), name
    assert np.array_equal(measure.view(np.uint64), want[1].view(np.uint64)), name
    assert np.array_equal(kth.view(np.uint32), want[2].view(np.uint32)), name


def test_static_knn_matches_handle_on_consecutive_calls(gd, cuda):
    import torch

    (cfg_a, p_a), (cfg_b, p_b) = _inputs(gd)
    dp_a, dp_b = gd.particles_to_device(p_a), gd.particles_to_device(p_b)
    want_a = _handle_knn(gd, cfg_a, dp_a)
    want_b = _handle_knn(gd, cfg_b, dp_b)
    out = [_outputs(cfg_a, len(p_a)), _outputs(cfg_b, len(p_b)), _outputs(cfg_a, len(p_a)),
           _outputs(cfg_b, len(p_b))]
    # the first call on the device does the one-time set-up
    gd.knn_static(cfg_a, dp_a, *out[0])
    gd.knn_static(cfg_b, dp_b, *out[1])
    torch.cuda.synchronize()
    _assert_same(out[0], want_a, "call 1 (3D, 65536)")
    _assert_same(out[1], want_b, "call 2 (2D, 50001)")
    # two warm calls in a row: no device memory taken or given back
    free_before = torch.cuda.mem_get_info()[0]
    gd.knn_static(cfg_a, dp_a, *out[2])
    gd.knn_static(cfg_b, dp_b, *out[3])
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    _assert_same(out[2], want_a, "call 3 (3D again)")
    _assert_same(out[3], want_b, "call 4 (2D again)")
    assert free_after == free_before


def test_static_knn_rejects_oversize_swarm(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    n = gd.STATIC_MAX_PARTICLES + 1
    cfg = workloads.config("c0_plain_small")
    dp = gd.particles_to_device(workloads.particles("c0_plain_small", n=n, seed=23))
    codes, measure, kth = _outputs(cfg, n)
    with pytest.raises(gd.GdError) as e:
        gd.knn_static(cfg, dp, codes, measure, kth)
    assert e.value.status == 5 and e.value.detail == n
    assert "65536" in e.value.message
    torch.cuda.synchronize()
    assert bool((codes == -7).all()) and bool((kth == -7.0).all())  # rejected before device work


def test_static_knn_reports_nonfinite_then_recovers(gd, cuda):
    import torch

    (cfg_a, p_a), _ = _inputs(gd)
    bad = p_a.copy()
    bad[4321, 1] = np.nan
    codes, measure, kth = _outputs(cfg_a, len(p_a))
    with pytest.raises(gd.GdError) as e:
        gd.knn_static(cfg_a, gd.particles_to_device(bad), codes, measure, kth)
    assert e.value.status == 3 and e.value.detail == 4321
    dp = gd.particles_to_device(p_a)
    gd.knn_static(cfg_a, dp, codes, measure, kth)
    torch.cuda.synchronize()
    _assert_same((codes, measure, kth), _handle_knn(gd, cfg_a, dp), "after the error")
