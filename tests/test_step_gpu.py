"""The Strang step's dynamics (gd_dynamics_step, gd_step) against the reference's own CUDA build.

oracle/_ref/step_<model>_<n>/ref_step runs the reference's dyn_rate_calc, diffusion_pos and
ssa_transport (or, with RADIATION, ssa_substep_1, the optical depth and ssa_substep_2), compiled
from the GameDev tree against the model header mod/make_models.py writes, in the order of its time
loop without the collision halves.  Both sides get the same particles and the same cuRAND streams
(curand_init(seed, i, 0)).  Errors are measured against each particle's own scales: angles
absolutely, the spherical radius relative to itself, angular momenta relative to the Keplerian
sqrt(G M R) and the radial speed relative to the Keplerian speed at R.  Bars:
  * t0 (3D, transport + diffusion, no radiation field): every step's dt and the clocks equal, every
    member of the cuRAND states identical (the same normal draws, in the same order), positions and
    velocities within 1e-12 of those scales;
  * c4 (3D, radiation pressure with Poynting-Robertson drag): the optical depth is a sum of FP64
    atomic deposits, whose order varies from run to run on both sides, so positions and velocities
    agree within 1e-9; dt, the clocks and the cuRAND states as above;
  * gd_step (collisions included): the clocks advance by the steps' dt, the represented dust mass
    is conserved to 1e-12, and the learned-radius search gives the same particles bit for bit as
    the plain search (its rows are the plain rows).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 65536


def _mass(p):
    return float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())


def _ours(gd, name, p, seed, steps):
    import torch

    from gamedev_b200 import workloads

    cfg = workloads.config(name)
    run = workloads.run_info(name)
    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(len(p), seed=seed)
    sw.set_clock(0.0, 0.0, run.dt_out)
    dts = []
    for _ in range(steps):
        sw.dynamics_step(run, dp, rng)
        dts.append(sw.clock()["dt"])
    torch.cuda.synchronize()
    out = dp.cpu().numpy()
    st = rng.cpu().numpy().reshape(len(p), -1)
    clk = sw.clock()
    sw.close()
    return out, st, dts, clk


def _scaled_errors(cfg, ours, ref):
    """Per-column errors on each particle's scales (see the module docstring)."""
    y = np.abs(ref[:, 1])
    R = np.maximum(y * np.abs(np.sin(ref[:, 2])), cfg.y_min)
    l_scale = np.sqrt(cfg.G * cfg.M_S * R)
    v_scale = np.sqrt(cfg.G * cfg.M_S / R)
    scales = [np.ones_like(y), np.maximum(y, cfg.y_min), np.ones_like(y), l_scale, v_scale, l_scale]
    return [np.abs(ours[:, c] - ref[:, c]) / scales[c] for c in range(6)]


def _compare(name, bar, steps=4):
    import gamedev_b200 as gd
    from gamedev_b200 import workloads
    from oracle.ref import refstep

    if not refstep.available(name, N):
        pytest.fail(f"oracle/_ref/step_{name}_{N} is missing: build the checker first (__graft_entry__.build)")
    cfg = workloads.config(name)
    p = workloads.particles(name, n=N)
    ours, st, dts, clk = _ours(gd, name, p, 3, steps)
    ref, rst, info = refstep.run(name, p, 3, steps, _mass(p))
    assert np.array_equal(np.array(dts).view(np.uint64), np.array(info["dt"]).view(np.uint64)), (dts, info["dt"])
    assert clk["clock_sim"] == info["clock_sim"] and clk["clock_out"] == info["clock_out"]
    # every member of each curandStateXORWOW (d, v[5], the two Box-Muller flags, the float and the
    # double spare); bytes 36-39 are alignment padding before the double, which copies need not keep
    members = np.r_[0:36, 40:48]
    assert np.array_equal(st[:, members], rst[:, members]), int((st[:, members] != rst[:, members]).any(axis=1).sum())
    for col, err in enumerate(_scaled_errors(cfg, ours, ref)):
        assert err.max() <= bar, (name, col, float(err.max()), int(np.argmax(err)))
    # grain sizes and counts are not the dynamics' to change
    assert np.array_equal(ours[:, 6:], p[:, 6:])
    moved = int((ours[:, 1] != p[:, 1]).sum())
    assert moved > 0.9 * N, moved
    return ours, ref


def test_transport_and_diffusion_match_reference_cuda(gd, cuda):
    _compare("t0_transport_3d", 1e-12)


def test_radiation_step_matches_reference_cuda(gd, cuda):
    _compare("c4_production_3d", 1e-9)


def test_full_step_conserves_mass_and_learned_search_changes_nothing(gd, cuda):
    import torch

    from gamedev_b200 import workloads

    name = "c4_production_3d"
    cfg = workloads.config(name)
    run = workloads.run_info(name)
    p = workloads.particles(name, n=N)
    mass = _mass(p)
    outs = []
    for learned in (False, True):
        sw = gd.SwarmCollision(cfg, N)
        dp = gd.particles_to_device(p)
        rng = gd.rngstate_init(N, seed=5)
        model = None
        if learned:
            # a briefly trained proposal: exactness does not depend on its quality
            codes, measure, kth = sw.knn(dp)
            feats = sw.radius_features(dp, kth, mass)
            model = gd.RadiusModel(cfg.R_0, seed=2)
            model.train(feats, kth, iterations=30, batch=4096, lr=2e-3)
            model.calibrate(feats, kth, 0.999)
            sw.invalidate_col_geometry()
        sw.set_clock(0.0, 0.0, run.dt_out)
        dts = []
        for _ in range(3):
            sw.step(run, dp, rng, mass, model)
            dts.append(sw.clock()["dt"])
        torch.cuda.synchronize()
        out = dp.cpu().numpy()
        clk = sw.clock()
        assert clk["steps"] == 3 and clk["clock_sim"] == pytest.approx(sum(dts), rel=1e-15)
        kept = out[:, 1] > 0  # particles still inside the domain
        m1 = float((out[:, 7] * math.pi * out[:, 6] ** 3 / 6.0)[kept].sum())
        m0 = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0)[kept].sum())
        assert abs(m1 - m0) <= 1e-12 * m0
        assert np.isfinite(out).all()
        outs.append(out)
        if model:
            model.close()
        sw.close()
    assert np.array_equal(outs[0].view(np.uint64), outs[1].view(np.uint64))


def test_captured_steps_equal_eager_steps(gd, cuda):
    """gd_step captured once into a CUDA graph (after one eager step) and replayed: the particles,
    the RNG streams and the clocks of eager steps, bit for bit; a non-finite particle written into
    the buffer before a replay is reported by gd_check_step with its index."""
    import torch

    from gamedev_b200 import workloads

    name = "t0_transport_3d"
    cfg = workloads.config(name)
    run = workloads.run_info(name)
    p = workloads.particles(name, n=N)
    mass = _mass(p)

    def fresh():
        sw = gd.SwarmCollision(cfg, N)
        dp = gd.particles_to_device(p)
        rng = gd.rngstate_init(N, seed=9)
        sw.set_clock(0.0, 0.0, run.dt_out)
        return sw, dp, rng

    sw, dp, rng = fresh()
    for _ in range(4):
        sw.step(run, dp, rng, mass)
    torch.cuda.synchronize()
    e_part = dp.cpu().numpy()
    e_uni = gd.rng_uniforms(rng, N, 4).cpu().numpy()
    e_clk = sw.clock()
    sw.close()

    sw, dp, rng = fresh()
    sw.step(run, dp, rng, mass)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sw.step(run, dp, rng, mass)
    for _ in range(3):
        graph.replay()
        sw.check_step()
    torch.cuda.synchronize()
    c_part = dp.cpu().numpy()
    c_uni = gd.rng_uniforms(rng, N, 4).cpu().numpy()
    c_clk = sw.clock()
    assert np.array_equal(e_part.view(np.uint64), c_part.view(np.uint64))
    assert np.array_equal(e_uni, c_uni)
    assert c_clk == e_clk and c_clk["steps"] == 4
    assert sw.last_operator_stats()["waves"] >= 2  # the replay's two operators

    dp[777, 1] = float("nan")
    graph.replay()
    with pytest.raises(gd.GdError) as e:
        sw.check_step()
    assert e.value.status == 3 and e.value.detail == 777
    del graph
    sw.close()
