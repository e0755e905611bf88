"""GPU parity of the frozen-bath collision operator against the CPU oracle.

Bars (written in the checks):
  * bath-start rate moments (col_bath_rate) within 2e-11 relative (the reference validator's bar
    for pair physics; 1e-8 for the ill-conditioned fragmentation moments): FP64 with device vs
    host transcendental functions, identical (count+1)/2 fold order;
  * one-wave operator: every owner's event count identical, grain size and count within 1e-12
    relative, and the device RNG advanced by exactly the number of deviates the oracle's replay of
    the same cuRAND stream consumed (checked bit for bit on the next deviate);
  * represented mass N_i m_i conserved per owner to 2e-12 and in total to 1e-12 relative;
  * a second operator on the stored rates: its bath-start moments equal a full re-rating bit for
    bit, and its chains the oracle's replay (K up to 96);
  * repeat runs bit-identical (the reference's run_chain.py hash check);
  * invalid input reported as a status, never a trap.
"""

import math

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

# pair-physics bar of the reference's own validator (val/swarm/src/validate_colphys.py:395-396):
# FP64 with device vs host transcendental functions, amplified by the (sl - ss) cancellations of
# the turbulent-speed regimes for near-equal grains
RATE_RTOL = 2e-11
# The jump moments of catastrophic fragmentation, 8 - (4L^2 + 8L) exp(-L)/(-expm1(-L)) and its
# first-moment analogue, cancel almost completely for L just above the 1e-3 series switch
# (_col_event.cuh:286-298): a last-bit difference between host and device exp/expm1 grows by
# ~1/L^2 there, so moment terms carry this looser bar.
MOMENT_RTOL = 1e-8
STATE_RTOL = 1e-12


def _setup(gd, cfg, p, seed=1):
    import torch

    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    sw.build_cache(dp)
    codes = torch.empty((len(p), cfg.n_k), dtype=torch.int32, device=dp.device)
    measure = torch.empty(len(p), dtype=torch.float64, device=dp.device)
    sw.get_cache(codes, measure)
    rng = gd.rngstate_init(len(p), seed=seed)
    site4, q, active = sw.get_sites()
    torch.cuda.synchronize()
    return sw, dp, rng, codes.cpu().numpy(), measure.cpu().numpy(), active.cpu().numpy()


def _one_wave(cfg):
    cfg.col_bath_max = 1.0e300
    cfg.col_bath_eps = 1.0e150
    return cfg


def _chain_cases(gd):
    from gamedev_b200 import workloads

    out = []
    cfg = cases.code_unit_config(gd, n_k=16, coag_kernel=0)
    out.append(("constant_kernel_3d", _one_wave(cfg), cases.random_swarm(cfg, 3000, 41), 3.0))
    cfg = cases.code_unit_config(gd, n_k=32, coag_kernel=1, three_d=False)
    out.append(("linear_kernel_2d", _one_wave(cfg), cases.random_swarm(cfg, 3000, 42), 3.0))
    cfg = cases.code_unit_config(gd, n_k=24, coag_kernel=2)
    out.append(("product_kernel_3d", _one_wave(cfg), cases.random_swarm(cfg, 2500, 43), 3.0))
    cfg = cases.code_unit_config(gd, n_k=32, coag_kernel=3)
    cfg.code_unit = 1
    cfg.v_frag = 3.0e-4
    cfg.init_smin = 1.0e-3
    out.append(("physical_kernel_code_units_frag", _one_wave(cfg), cases.random_swarm(cfg, 3000, 44), 3.0))
    cfg = workloads.config("c0_plain_small")
    out.append(("c0_physical_units", _one_wave(cfg), workloads.particles("c0_plain_small", n=4000), 3.0))
    cfg = workloads.config("c1_multisize_2d")
    out.append(("c1_frag_2d", _one_wave(cfg), workloads.particles("c1_multisize_2d", n=4000), 3.0))
    return out


def _calibrated_duration(oracle_lib, cfg, p, codes, measure, active, events_per_owner):
    lam = len(p) / cfg.n_k / _total_mass(p)
    cached, rate, _, _ = oracle_lib.bath_rate(cfg, p, codes, measure, active, p[:, 6], p[:, 7], lam)
    r = rate[active.astype(bool) & (rate > 0)]
    # the fastest owner expects `events_per_owner` events; slower owners proportionally fewer
    return events_per_owner / float(r.max()), lam, cached


def _total_mass(p):
    return float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())


@pytest.mark.parametrize("idx", range(6))
def test_operator_one_wave_matches_oracle_chain(gd, cuda, oracle_lib, idx):
    import torch

    name, cfg, p, evpo = _chain_cases(gd)[idx]
    sw, dp, rng, codes, measure, active = _setup(gd, cfg, p)
    duration, lam, cached_o = _calibrated_duration(oracle_lib, cfg, p, codes, measure, active, evpo)
    # total dust mass enters lambda_0 exactly as the caller passes it
    mass = _total_mass(p)
    U = gd.rng_uniforms(rng, len(p), 96).cpu().numpy()
    sw.evolve_local_collisions(dp, rng, duration, mass)
    stats = sw.last_operator_stats()
    assert stats["waves"] == 1, stats
    cached, time_g, events_g, size_old, numr_old = (t.cpu().numpy() for t in sw.owner_state())
    out = dp.cpu().numpy()
    nxt = gd.rng_uniforms(rng, len(p), 1).cpu().numpy()[:, 0]
    torch.cuda.synchronize()

    # bath-start moments
    act = active.astype(bool)
    np.testing.assert_allclose(cached[act][:, [0, 3]], cached_o[act][:, [0, 3]], rtol=RATE_RTOL, atol=0, err_msg=name)
    np.testing.assert_allclose(cached[act][:, 1:3], cached_o[act][:, 1:3], rtol=MOMENT_RTOL, atol=0, err_msg=name)

    n_events = 0
    for i in np.nonzero(act)[0]:
        err, st, used = oracle_lib.chain_owner(cfg, int(i), p, codes, measure, active, p[:, 6].copy(),
                                               p[:, 7].copy(), lam, duration, cached_o[i], U[i])
        assert err == 0, (name, i, err)
        assert int(st[7]) == events_g[i], (name, i, st[7], events_g[i])
        n_events += int(st[7])
        assert math.isclose(st[0], out[i, 6], rel_tol=STATE_RTOL), (name, i, st[0], out[i, 6])
        assert math.isclose(st[1], out[i, 7], rel_tol=STATE_RTOL), (name, i)
        assert st[2] == time_g[i]
        # the device stream advanced by exactly `used` deviates
        assert nxt[i] == U[i, used], (name, i, used)
    assert n_events > 0, name
    assert stats["events"] == n_events
    # mass: per owner and in total
    m0 = p[:, 7] * p[:, 6] ** 3
    m1 = out[:, 7] * out[:, 6] ** 3
    assert (np.abs(m1 - m0) <= 2e-12 * np.maximum(m0, m1)).all()
    assert abs(m1.sum() - m0.sum()) <= 1e-12 * m0.sum()
    sw.close()


@pytest.mark.parametrize("idx", range(6))
def test_bath_rates_match_oracle(gd, cuda, oracle_lib, idx):
    """gd_bath_rates (col_bath_rate alone, eager) against the oracle's bath rate on the current
    particles as reservoir, and against the operator's own bath-start moments bit for bit."""
    name, cfg, p, _ = _chain_cases(gd)[idx]
    sw, dp, rng, codes, measure, active = _setup(gd, cfg, p)
    mass = _total_mass(p)
    lam = len(p) / cfg.n_k / mass
    cached_o, _, _, _ = oracle_lib.bath_rate(cfg, p, codes, measure, active, p[:, 6], p[:, 7], lam)
    got = sw.bath_rates(dp, mass).cpu().numpy()
    act = active.astype(bool)
    np.testing.assert_allclose(got[act][:, [0, 3]], cached_o[act][:, [0, 3]], rtol=RATE_RTOL, atol=0, err_msg=name)
    np.testing.assert_allclose(got[act][:, 1:3], cached_o[act][:, 1:3], rtol=MOMENT_RTOL, atol=0, err_msg=name)
    # the operator's tick-0 rates are the same kernel on the same reservoir: the same bits
    sw.evolve_local_collisions(dp, rng, 1.0e-30, mass)
    op = sw.owner_state()[0].cpu().numpy()
    assert np.array_equal(got[act].view(np.uint64), op[act].view(np.uint64)), name
    sw.close()


@pytest.mark.parametrize("idx", range(6))
def test_bath_chain_equals_the_one_wave_operator(gd, cuda, oracle_lib, idx):
    """gd_bath_chain (one frozen bath for every owner, launched eagerly) leaves the particles and the
    RNG streams bit for bit as the one-wave operator of the same duration does, with the same event
    count: the same rates, skip scan and chain outside the operator's graph."""
    import torch

    name, cfg, p, evpo = _chain_cases(gd)[idx]
    sw, dp, rng, codes, measure, active = _setup(gd, cfg, p)
    duration, _, _ = _calibrated_duration(oracle_lib, cfg, p, codes, measure, active, evpo)
    mass = _total_mass(p)
    dp2, rng2 = dp.clone(), rng.clone()
    sw.evolve_local_collisions(dp, rng, duration, mass)
    stats = sw.last_operator_stats()
    assert stats["waves"] == 1, stats
    events = sw.bath_chain(dp2, rng2, mass, duration)
    torch.cuda.synchronize()
    assert events == stats["events"] and events > 0, (name, events, stats["events"])
    assert np.array_equal(dp2.cpu().numpy().view(np.uint64), dp.cpu().numpy().view(np.uint64)), name
    assert torch.equal(rng2.cpu(), rng.cpu()), name
    # a second bath from the advanced state runs too (the call keeps no state of its own)
    assert sw.bath_chain(dp2, rng2, mass, duration) >= 0
    sw.close()


def test_operator_repeat_is_bit_identical_and_multiwave(gd, cuda):
    """Full controller (moving bins, merged bins, many waves): two runs from the same state give
    byte-identical particles and RNG states, and represented mass is conserved."""
    import torch

    from gamedev_b200 import workloads

    cfg = workloads.config("c1_multisize_2d")
    p = workloads.particles("c1_multisize_2d", n=20000)
    mass = _total_mass(p)
    results = []
    for _ in range(2):
        sw, dp, rng, *_ = _setup(gd, cfg, p, seed=5)
        sw.evolve_local_collisions(dp, rng, 1.0e-9 * workloads.orbital_time(), mass)
        rate_max = float(sw.owner_state()[0][:, 0].max().item())
        dp.copy_(gd.particles_to_device(p))
        rng = gd.rngstate_init(len(p), seed=5)
        for _ in range(3):
            # ~20 expected events for the fastest owner: the change bounds split it into many waves
            sw.evolve_local_collisions(dp, rng, 20.0 / rate_max, mass)
        torch.cuda.synchronize()
        results.append((dp.cpu().numpy().copy(), rng.cpu().numpy().copy(), sw.last_operator_stats()))
        sw.close()
    (a, ra, sa), (b, rb, sb) = results
    assert np.array_equal(a, b)
    # RNG states compared as streams: struct padding bytes of curandState are not preserved by
    # member-wise copies, so equal states need not be equal byte strings
    import torch as _t

    ua = gd.rng_uniforms(_t.from_numpy(ra).cuda(), len(p), 4).cpu().numpy()
    ub = gd.rng_uniforms(_t.from_numpy(rb).cuda(), len(p), 4).cpu().numpy()
    assert np.array_equal(ua, ub)
    assert sa["waves"] >= 1
    m0 = (p[:, 7] * p[:, 6] ** 3).sum()
    assert abs((a[:, 7] * a[:, 6] ** 3).sum() - m0) <= 1e-12 * m0


def test_operator_rejects_nonfinite_state(gd, cuda):
    """A non-finite grain count is reported as a status (screen or controller), never a trap."""
    import torch

    cfg = cases.code_unit_config(gd, n_k=16, coag_kernel=0)
    p = cases.random_swarm(cfg, 2000, 61)
    sw, dp, rng, *_ = _setup(gd, cfg, p)
    bad = dp.clone()
    bad[123, 7] = float("nan")
    with pytest.raises(gd.GdError) as e:
        sw.evolve_collisions(bad, rng, 1.0, _total_mass(p))
    assert e.value.status == 3 and e.value.detail == 123  # GD_ERR_NONFINITE, the reference's exit path
    with pytest.raises(gd.GdError) as e:
        sw.evolve_local_collisions(bad, rng, 1.0, _total_mass(p))
    assert e.value.status in (4, 8)  # chain error or invalid controller state
    # the handle recovers on valid input
    sw.evolve_local_collisions(dp, rng, 1.0e-3, _total_mass(p))
    torch.cuda.synchronize()


def test_operator_rejects_invalid_arguments(gd, cuda):
    cfg = cases.code_unit_config(gd, n_k=8)
    p = cases.random_swarm(cfg, 500, 62)
    sw, dp, rng, *_ = _setup(gd, cfg, p)
    with pytest.raises(gd.GdError) as e:
        sw.evolve_local_collisions(dp, rng, float("nan"), 1.0)
    assert e.value.status == 1
    with pytest.raises(gd.GdError) as e:
        sw.evolve_local_collisions(dp, rng, 1.0, -1.0)
    assert e.value.status == 1


@pytest.mark.parametrize("idx", range(6))
def test_pair_rates_match_oracle(gd, cuda, oracle_lib, idx):
    """Every (owner, slot) term the bath-start fold sums, device vs oracle (RATE_RTOL relative)."""
    import torch

    name, cfg, p, _ = _chain_cases(gd)[idx]
    sw, dp, rng, codes, measure, active = _setup(gd, cfg, p)
    mass = _total_mass(p)
    lam = len(p) / cfg.n_k / mass
    ids = np.nonzero(active)[0][:600].astype(np.int32)
    got = sw.pair_rates(dp, torch.from_numpy(ids).cuda(), mass).cpu().numpy()
    tol = np.array([RATE_RTOL, MOMENT_RTOL, MOMENT_RTOL, RATE_RTOL, RATE_RTOL])
    bad = []
    for a, i in enumerate(ids):
        want = np.zeros((cfg.n_k, 5))
        equal = np.zeros(cfg.n_k, dtype=bool)
        for s_ in range(cfg.n_k):
            c = codes[i, s_]
            if c >= 0 and measure[i] > 0:
                j = c // 3
                r, v = oracle_lib.pair_rate(cfg, p[i, 1], p[i, 2], p[j, 1], p[j, 2], p[i, 6], p[j, 6], p[j, 7], lam,
                                            measure[i])
                f, mean, sec, mx = oracle_lib.outcome_moments(cfg, p[i, 6], p[j, 6], v >= cfg.v_frag)
                r *= f
                want[s_] = [r, r * mean, r * sec, mx if r > 0 else 0.0, v]
                equal[s_] = p[i, 6] == p[j, 6]
        # Identical grains (the owner's own slot, or an equal-size partner): the drift speed is the
        # rounding residual of one fused multiply-add, so the term is noise at the 1e-16 level of
        # the owner's other terms.  It is held to an absolute bar on the owner's row sums, and its
        # maximum (which follows the sign of that residual) is not compared.
        scale = np.abs(want).sum(axis=0) * tol
        scale[4] = np.abs(want[:, 4]).max() * RATE_RTOL
        for s_ in range(cfg.n_k):
            g, w = got[a, s_], want[s_]
            if equal[s_]:
                ok = np.all((np.abs(g - w) <= scale)[[0, 1, 2, 4]])
            else:
                ok = np.all((g == w) | (np.abs(g - w) <= tol * np.maximum(np.abs(g), np.abs(w))))
            if not ok:
                bad.append((int(i), s_, int(codes[i, s_]), float(measure[i]), g, w))
    if bad:
        lines = [f"{name}: {len(bad)} of {len(ids) * cfg.n_k} pairs differ"]
        for i, s_, c, mv, g, w in bad[:4]:
            j = c // 3
            lines.append(f"owner {i} slot {s_} code {c} measure {mv:.17g} si {p[i, 6]:.17g} sj {p[j, 6]:.17g}")
            lines.append("  gpu    " + " ".join(f"{v:.17g}" for v in g))
            lines.append("  oracle " + " ".join(f"{v:.17g}" for v in w))
        pytest.fail("\n".join(lines))


def _controller_valid(data: dict) -> bool:
    """The checks the reference's validator applies to an archived controller summary
    (val/swarm/src/run_chain.py:99-170, validate_controller), restated."""
    numeric = ("minimum_duration", "maximum_duration", "minimum_limit_scale", "maximum_f", "maximum_e",
               "maximum_touched", "maximum_events", "maximum_g", "maximum_g_upper", "maximum_d_bath")
    baths = data.get("baths", [])
    finite = all(math.isfinite(float(data.get(k, math.nan))) for k in numeric)
    complete = (data.get("schema") == 2 and data.get("bath_count") == len(baths) and data.get("bath_count", 0) > 0
                and data.get("operator_count", 0) > 0 and data.get("wave_count", 0) > 0
                and data.get("persistent_overshoots") == 0)
    continuation = data.get("continuation_launches", 0) > 0
    bath_numeric = ("duration", "limit_before", "limit_after", "max_f", "max_e", "max_touched", "max_events",
                    "max_g", "max_g_upper", "d_bath")
    records = all(r.get("operator", 0) > 0 and r.get("bath", 0) > 0 and r.get("merged_bins", 0) > 0
                  and r.get("group", -1) >= 0 and r.get("duration", 0.0) > 0.0
                  and 0.25 <= r.get("limit_before", 0.0) <= 1.0 and 0.25 <= r.get("limit_after", 0.0) <= 1.0
                  and all(math.isfinite(float(r.get(k, math.nan))) for k in bath_numeric)
                  and all(r.get(k, -1.0) >= 0.0 for k in bath_numeric if k != "limit_before")
                  and not r.get("persistent_overshoot", True) for r in baths)
    return finite and complete and continuation and records


def _controller_equivalent(a, b) -> bool:
    """The validator's repeat comparison (run_chain.py:64-96): equal keys and structure, numbers
    within 1e-12 relative or absolute (atomic-sum roundoff)."""
    if isinstance(a, dict):
        return isinstance(b, dict) and a.keys() == b.keys() and all(_controller_equivalent(a[k], b[k]) for k in a)
    if isinstance(a, list):
        return isinstance(b, list) and len(a) == len(b) and all(_controller_equivalent(x, y) for x, y in zip(a, b))
    if isinstance(a, (int, float)) and not isinstance(a, bool):
        return (isinstance(b, (int, float)) and not isinstance(b, bool)
                and math.isclose(float(a), float(b), rel_tol=1e-12, abs_tol=1e-12))
    return a == b


def test_controller_summary_passes_reference_validator(gd, cuda):
    """COL_DIAGNOSTICS summary (gd_controller_summary) of a multi-wave run: accepted by the checks of
    the reference's run_chain.py validator, repeat-consistent under its comparison, and cleared by
    gd_reset_controller as at an output boundary."""
    import torch

    from gamedev_b200 import workloads

    cfg = workloads.config("c1_multisize_2d")
    p = workloads.particles("c1_multisize_2d", n=20000)
    mass = _total_mass(p)
    summaries = []
    for _ in range(2):
        sw, dp, rng, *_ = _setup(gd, cfg, p, seed=5)
        sw.evolve_local_collisions(dp, rng, 1.0e-9 * workloads.orbital_time(), mass)
        rate_max = float(sw.owner_state()[0][:, 0].max().item())
        sw.reset_controller()
        dp.copy_(gd.particles_to_device(p))
        rng = gd.rngstate_init(len(p), seed=5)
        for _ in range(3):
            sw.evolve_local_collisions(dp, rng, 20.0 / rate_max, mass)
        torch.cuda.synchronize()
        summaries.append(sw.controller_summary())
        sw.reset_controller()
        empty = sw.controller_summary()
        assert empty["operator_count"] == 0 and empty["baths"] == []
        sw.close()
    a, b = summaries
    assert a["operator_count"] == 3 and a["wave_count"] > 3 and a["bath_count"] > 3
    assert _controller_valid(a)
    assert _controller_equivalent(a, b)


@pytest.mark.parametrize("n_k,coag_kernel,three_d", [(24, 2, True), (64, 3, True), (96, 3, True), (96, 1, False)])
def test_second_operator_on_stored_rates(gd, cuda, oracle_lib, n_k, coag_kernel, three_d):
    """Two one-wave operators on one neighbour cache.  The second rates its owners through the
    stored pairs: an owner whose reservoir entry changed in the first is evaluated whole, one whose
    partners changed re-evaluates only those pairs and is folded again, the rest keep their rates.
    Its bath-start moments equal a full re-rating of the same state (gd_bath_rates) bit for bit, and
    its chains leave every owner as the oracle's replay from the first operator's result.  K = 96
    takes the planner's row rescan and the shared-memory fold (K above 64, not a power of two)."""
    cfg = _one_wave(cases.code_unit_config(gd, n_k=n_k, coag_kernel=coag_kernel, three_d=three_d))
    p = cases.random_swarm(cfg, 3000, 50 + n_k)
    sw, dp, rng, codes, measure, active = _setup(gd, cfg, p)
    duration, lam, _ = _calibrated_duration(oracle_lib, cfg, p, codes, measure, active, 3.0)
    mass = _total_mass(p)
    sw.evolve_local_collisions(dp, rng, duration, mass)
    first = sw.last_operator_stats()
    assert first["waves"] == 1 and first["events"] > 0, first
    p1 = dp.cpu().numpy()
    full = sw.bath_rates(dp, mass).cpu().numpy()
    # the second operator sized as the first on the grown grains: 3 expected events for the
    # fastest owner at its bath start
    duration = 3.0 / float(full[active.astype(bool), 0].max())
    U = gd.rng_uniforms(rng, len(p), 512).cpu().numpy()
    sw.evolve_local_collisions(dp, rng, duration, mass)
    stats = sw.last_operator_stats()
    assert stats["waves"] == 1, stats
    cached, time_g, events_g, _, _ = (t.cpu().numpy() for t in sw.owner_state())
    out = dp.cpu().numpy()
    nxt = gd.rng_uniforms(rng, len(p), 1).cpu().numpy()[:, 0]
    act = active.astype(bool)
    # the second operator's bath-start moments, from stored and re-evaluated pairs, against a full
    # re-rating of the same reservoir
    assert np.array_equal(cached[act].view(np.uint64), full[act].view(np.uint64))
    changed = (p1[:, 6] != p[:, 6]) | (p1[:, 7] != p[:, 7])
    assert changed.any() and not changed.all()
    cached_o, _, _, _ = oracle_lib.bath_rate(cfg, p1, codes, measure, active, p1[:, 6], p1[:, 7], lam)
    n_events = 0
    for i in np.nonzero(act)[0]:
        err, st, used = oracle_lib.chain_owner(cfg, int(i), p1, codes, measure, active, p1[:, 6].copy(),
                                               p1[:, 7].copy(), lam, duration, cached_o[i], U[i])
        assert err == 0, (n_k, i, err)
        assert int(st[7]) == events_g[i], (n_k, i, st[7], events_g[i])
        n_events += int(st[7])
        assert math.isclose(st[0], out[i, 6], rel_tol=STATE_RTOL), (n_k, i, st[0], out[i, 6])
        assert math.isclose(st[1], out[i, 7], rel_tol=STATE_RTOL), (n_k, i)
        assert nxt[i] == U[i, used], (n_k, i, used)
    assert stats["events"] == n_events
    sw.close()
