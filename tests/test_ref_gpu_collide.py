"""The B200 collision operator against the reference's own CUDA collision build on the same GPU.

oracle/_ref/collide_<model>_<n>/ref_collide runs the reference's evolve_collisions glue and
evolve_local_collisions with its kernels, compiled from the GameDev tree (oracle/ref/Makefile)
against the model header mod/make_models.py writes for the same configuration.  Both sides get the
same particles, the same cuRAND seed (curand_init(seed, i, 0)) and the same operator length.

Bars:
  * Morton search (c1 shapes: 2D, fragmentation): the reference writes neighbour lists in the same
    ascending (d^2, code) order, so the event chains are the same: every particle's grain size and
    count after the operator equal the reference's to 1e-12 relative, over thousands of events;
  * KD search (c0 shapes: 3D, coagulation): the reference's lists are in heap order, so a chain can
    pick a different partner for the same draw.  Across 16 seeds:
      - M_0 (M_k = sum N_i m_i^k) agrees within 1%, and M_1 (the dust mass) to 1e-12;
      - M_2 passes a two-sample Mann-Whitney test on the per-seed values (p > 0.01).  A 1% bar on
        M_2 is out of reach for any implementation here: runaway growth from monodisperse grains
        makes the per-seed M_2 spread by 80-200% (relative SD), for the reference as much as for
        this build;
      - a two-sample KS test on the mass-weighted log grain size gives p > 0.01;
      - in each run at least 90% of the particles still come out identical (a different partner
        order changes only the owners it reaches).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 65536


def _refc():
    from oracle.ref import refcollide

    return refcollide


def _mass(p):
    return float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())


def _duration(gd, cfg, p, events_fastest):
    """Operator length giving the fastest owner `events_fastest` expected events at bath start."""
    from gamedev_b200 import workloads

    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(len(p), seed=1)
    sw.evolve_collisions(dp, rng, 1.0e-12 * workloads.orbital_time(), _mass(p))
    rates = sw.owner_state()[0][:, 0].cpu().numpy()
    sw.close()
    return events_fastest / rates.max()


def _ours(gd, cfg, p, seed, duration):
    import torch

    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(len(p), seed=seed)
    sw.evolve_collisions(dp, rng, duration, _mass(p))
    torch.cuda.synchronize()
    out = dp.cpu().numpy()
    stats = sw.last_operator_stats()
    sw.close()
    return out, stats


def _moment(p, k):
    return float((p[:, 7] * (math.pi * p[:, 6] ** 3 / 6.0) ** k).sum())


def _weighted_ks(xa, wa, xb, wb):
    """Two-sample KS statistic of weighted samples and its asymptotic p-value, with the Kish
    effective sample sizes (sum w)^2 / sum w^2."""
    grid = np.sort(np.concatenate([xa, xb]))
    def ecdf(x, w):
        o = np.argsort(x)
        cw = np.cumsum(w[o]) / w.sum()
        return np.concatenate([[0.0], cw])[np.searchsorted(x[o], grid, side="right")]
    d = float(np.abs(ecdf(xa, wa) - ecdf(xb, wb)).max())
    na = wa.sum() ** 2 / (wa ** 2).sum()
    nb = wb.sum() ** 2 / (wb ** 2).sum()
    en = math.sqrt(na * nb / (na + nb))
    lam = (en + 0.12 + 0.11 / en) * d
    p = 2.0 * sum((-1) ** (j - 1) * math.exp(-2.0 * j * j * lam * lam) for j in range(1, 101))
    return d, min(1.0, max(0.0, p))


def test_morton_operator_matches_reference_cuda_per_particle(gd, cuda):
    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c1_multisize_2d"
    if not refcollide.available(model, N):
        pytest.skip("oracle/_ref reference collision build absent (reference tree not mounted at build time)")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=11)
    rates_duration = _duration(gd, cfg, p, 2000.0)
    for seed in (1, 2):
        ours, stats = _ours(gd, cfg, p, seed, rates_duration)
        ref, info = refcollide.run(model, p, seed, rates_duration, _mass(p), 1, timeout=600)
        same = (np.isclose(ours[:, 6], ref[:, 6], rtol=1e-12, atol=0)
                & np.isclose(ours[:, 7], ref[:, 7], rtol=1e-12, atol=0))
        assert same.all(), (seed, int((~same).sum()), stats)
        assert stats["events"] > 1000, stats
        # several waves: every wave after the first re-rates only the owners and pairs whose
        # reservoir entries changed (the stored-pair path), against the reference's full rating
        assert stats["waves"] > 1, stats
        assert abs(_moment(ours, 1) - _mass(p) * 1.0) <= 1e-12 * _mass(p)


def test_kd_operator_matches_reference_cuda_statistically(gd, cuda):
    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c0_plain_small"
    if not refcollide.available(model, N):
        pytest.skip("oracle/_ref reference collision build absent (reference tree not mounted at build time)")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=12)
    from scipy.stats import mannwhitneyu

    d = _duration(gd, cfg, p, 10.0)
    mo, mr = np.zeros(3), np.zeros(3)
    m2o, m2r = [], []
    xo, wo, xr, wr = [], [], [], []
    for seed in range(1, 17):
        ours, _ = _ours(gd, cfg, p, seed, d)
        ref, _ = refcollide.run(model, p, seed, d, _mass(p), 1, timeout=600)
        same = np.isclose(ours[:, 6], ref[:, 6], rtol=1e-12, atol=0) & np.isclose(ours[:, 7], ref[:, 7], rtol=1e-12)
        assert same.mean() >= 0.9, (seed, float(same.mean()))
        for k in range(3):
            mo[k] += _moment(ours, k)
            mr[k] += _moment(ref, k)
        m2o.append(_moment(ours, 2))
        m2r.append(_moment(ref, 2))
        for arr, xs, ws in ((ours, xo, wo), (ref, xr, wr)):
            xs.append(np.log(arr[:, 6]))
            ws.append(arr[:, 7] * arr[:, 6] ** 3)  # mass weight
    assert abs(mo[0] / mr[0] - 1.0) < 0.01, mo / mr
    assert abs(mo[1] / mr[1] - 1.0) < 1e-12, mo / mr
    assert mannwhitneyu(m2o, m2r).pvalue > 0.01, (m2o, m2r)
    dstat, pval = _weighted_ks(np.concatenate(xo), np.concatenate(wo), np.concatenate(xr), np.concatenate(wr))
    assert pval > 0.01, (dstat, pval)


def test_morton_controller_summary_matches_reference(gd, cuda):
    """COL_DIAGNOSTICS: over two operators on the Morton shapes (the same event chains as the
    reference), the controller summary gd_controller_summary returns equals the one the reference's
    COL_DIAGNOSTICS build writes (save_col_controller): operator, bath and wave counts, overshoot
    counts and flags, every bath's group, merged bins, duration and limit scale before and after
    exactly; the audit maxima, sums of FP64 atomics in either build, to 1e-9 relative (1e-12
    absolute where they cancel).  Chain
    launches per wave are not compared: this build's chain is persistent (one launch per wave)
    where the reference relaunches chains capped at COL_EVENT_CAP events."""
    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c1_multisize_2d"
    if not refcollide.available(model, N, diagnostics=True):
        pytest.skip("oracle/_ref reference COL_DIAGNOSTICS build absent (reference tree not mounted at build time)")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=11)
    d = _duration(gd, cfg, p, 2000.0)
    import torch

    sw = gd.SwarmCollision(cfg, N)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(N, seed=1)
    for _ in range(2):
        sw.evolve_collisions(dp, rng, d, _mass(p))
    torch.cuda.synchronize()
    ours = sw.controller_summary()
    sw.close()
    _, info = refcollide.run(model, p, 1, d, _mass(p), 2, timeout=600, diagnostics=True)
    ref = info["summary"]
    exact = ["schema", "operator_count", "bath_count", "wave_count", "activity_overshoots",
             "distribution_overshoots", "persistent_overshoots", "minimum_duration", "maximum_duration",
             "minimum_limit_scale"]
    for key in exact:
        assert ours[key] == ref[key], (key, ours[key], ref[key])
    close = ["maximum_f", "maximum_e", "maximum_touched", "maximum_events", "maximum_g", "maximum_g_upper",
             "maximum_d_bath"]
    for key in close:
        assert math.isclose(ours[key], ref[key], rel_tol=1e-9, abs_tol=1e-12), (key, ours[key], ref[key])
    assert ours["bath_count"] > 2 and ours["wave_count"] >= 2
    assert len(ours["baths"]) == len(ref["baths"])
    for a, b in zip(ours["baths"], ref["baths"]):
        for key in ("operator", "group", "bath", "merged_bins", "duration", "limit_before", "limit_after",
                    "activity_overshoot", "distribution_overshoot", "persistent_overshoot"):
            assert a[key] == b[key], (key, a, b)
        for key in ("max_f", "max_e", "max_touched", "max_events", "max_g", "max_g_upper", "d_bath"):
            # d_bath is a difference of audit sums: where it cancels, the residual is ~1e-17 in one
            # summation order and 0 in another
            assert math.isclose(a[key], b[key], rel_tol=1e-9, abs_tol=1e-12), (key, a, b)


def test_morton_event_categories_match_reference(gd, cuda):
    """COL_DIAGNOSTICS event bookkeeping: per operator, the events per outcome category and their
    summed log mass change (gd_event_totals) equal the event_counts and event_log_mass_sums of the
    reference's per-operator diagnostics log, on the Morton shapes where the event chains are the
    same: counts exactly, log-mass sums to 1e-9 relative (summation order)."""
    import torch

    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c1_multisize_2d"
    if not refcollide.available(model, N, diagnostics=True):
        pytest.skip("oracle/_ref reference COL_DIAGNOSTICS build absent (reference tree not mounted at build time)")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=11)
    d = _duration(gd, cfg, p, 2000.0)
    sw = gd.SwarmCollision(cfg, N)
    sw.set_diagnostics(True)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(N, seed=1)
    ours = []
    for _ in range(2):
        sw.evolve_collisions(dp, rng, d, _mass(p))
        torch.cuda.synchronize()
        ours.append(sw.event_totals())
    sw.close()
    _, info = refcollide.run(model, p, 1, d, _mass(p), 2, timeout=600, diagnostics=True)
    log = info["operator_log"]
    assert len(log) == 2
    for (counts, lm), line in zip(ours, log):
        assert [int(c) for c in counts] == [int(c) for c in line["event_counts"]], (counts, line["event_counts"])
        assert int(counts.sum()) > 1000
        for a, b in zip(lm, line["event_log_mass_sums"]):
            assert math.isclose(float(a), float(b), rel_tol=1e-9, abs_tol=1e-12), (lm, line["event_log_mass_sums"])


def test_operator_log_equals_reference_log(gd, cuda):
    """The per-operator COL_DIAGNOSTICS log (gd_operator_log) against the reference's
    collision_local_*.jsonl on the Morton shapes, where the event chains are the same: per operator
    its number, duration, waves, owner updates, finest ticks and event counts exactly; per group its
    owners, final and initial levels, bath length, binding constraint, coarsened / refined /
    constrained updates, updates, overshoots and persistent overshoots exactly; the requested
    lengths, the oldest linked reservoir and the bath length over request to 1e-12 (FP64 atomic
    rate-bin sums), the growth and predicted-activity maxima to 1e-9 (FP64 atomic audit sums).
    Chain blocks and launches count this build's persistent chain, and the seconds are device time:
    present and non-negative."""
    import torch

    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c1_multisize_2d"
    if not refcollide.available(model, N, diagnostics=True):
        pytest.fail("oracle/_ref reference COL_DIAGNOSTICS build absent: build the checker first")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=11)
    d = _duration(gd, cfg, p, 2000.0)
    sw = gd.SwarmCollision(cfg, N)
    sw.set_diagnostics(True)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(N, seed=1)
    for _ in range(2):
        sw.evolve_collisions(dp, rng, d, _mass(p))
    torch.cuda.synchronize()
    ours = sw.operator_log()
    sw.close()
    _, info = refcollide.run(model, p, 1, d, _mass(p), 2, timeout=600, diagnostics=True)
    ref = info["operator_log"]
    assert len(ours) == len(ref) == 2
    exact_top = ("schema", "method", "operator", "duration", "waves", "owner_updates", "finest_ticks", "event_counts")
    exact_group = ("id", "owners", "level", "dt", "initial_level", "coarsened_updates", "refined_updates",
                   "neighbor_constrained_updates", "initial_binding_constraint", "updates", "overshoots",
                   "persistent_overshoots")
    # the requested lengths come from FP64 atomic rate-bin sums: their last bits follow the sum order
    # on both sides, while the power-of-two levels and bath lengths built from them agree exactly
    close_group = {"minimum_requested_dt": 1e-12, "maximum_requested_dt": 1e-12, "final_requested_dt": 1e-12,
                   "initial_requested_dt": 1e-12, "max_snapshot_age_at_start": 1e-12,
                   "max_requested_dt_ratio": 1e-12, "max_growth": 1e-9, "max_predicted_activity": 1e-9}
    assert set(ours[0]) == set(ref[0])
    for a, b in zip(ours, ref):
        for key in exact_top:
            assert a[key] == b[key], (key, a[key], b[key])
        for key in ("chain_blocks", "chain_launches", "chain_seconds", "audit_seconds", "scheduler_wall_seconds"):
            assert a[key] >= 0
        assert a["waves"] > 1
        assert len(a["groups"]) == len(b["groups"])
        for ga, gb in zip(a["groups"], b["groups"]):
            assert set(ga) == set(gb)
            for key in exact_group:
                assert ga[key] == gb[key], (ga["id"], key, ga[key], gb[key])
            for key, tol in close_group.items():
                assert math.isclose(ga[key], gb[key], rel_tol=tol, abs_tol=1e-15), (ga["id"], key, ga[key], gb[key])
        for x, y in zip(a["event_log_mass_sums"], b["event_log_mass_sums"]):
            assert math.isclose(x, y, rel_tol=1e-9, abs_tol=1e-12)
    assert sum(g["updates"] for g in ours[0]["groups"]) > 3


def _bootstrap_ratio(a, b, reps=4000, seed=0):
    """Ratio of the means of two per-seed samples and its 95% bootstrap interval (seeds resampled
    independently on each side)."""
    rng = np.random.default_rng(seed)
    a, b = np.asarray(a), np.asarray(b)
    ra = rng.integers(0, len(a), (reps, len(a)))
    rb = rng.integers(0, len(b), (reps, len(b)))
    ratios = a[ra].mean(axis=1) / b[rb].mean(axis=1)
    return float(a.mean() / b.mean()), float(np.quantile(ratios, 0.025)), float(np.quantile(ratios, 0.975))
