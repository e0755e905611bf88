"""Generate the golden vectors committed beside this script.

Two sources, both the reference itself:
  colphys_golden.json   the reference's independent Python pair-velocity formulas
                        (val/swarm/src/validate_colphys.py: turbulent_velocity, brownian_velocity,
                        local_pair_velocity), imported from the GameDev tree, over all six
                        Ormel-Cuzzi regimes in physical and code units;
  ref_host_golden.json  the reference's own collision headers compiled on the host
                        (oracle/_ref, built by oracle/ref/Makefile): pair rates, outcome moments and
                        samples, ball measures, size-bin merging, bath durations, audits and the
                        power-of-two scheduler.

Run in a tree where the reference is mounted:  python tests/golden/make_golden.py [reference root]
"""

from __future__ import annotations

import importlib.util
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def colphys(reference: Path):
    spec = importlib.util.spec_from_file_location("validate_colphys",
                                                  reference / "val/swarm/src/validate_colphys.py")
    vc = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(vc)
    rng = np.random.default_rng(2024)
    rows = []
    for code_unit in (False, True):
        for _ in range(240):
            radius = float(rng.uniform(0.6, 1.4))
            height = float(rng.uniform(-0.08, 0.08) * radius)
            si = float(math.exp(rng.uniform(math.log(1e-9), math.log(50.0))))
            sj = float(math.exp(rng.uniform(math.log(1e-9), math.log(50.0))))
            if rng.uniform() < 0.1:
                sj = si
            zero = np.zeros(3)
            _, speed = vc.local_pair_velocity(zero, zero, si, sj, radius, height, code_unit)
            rows.append({"radius": radius, "height": height, "size_i": si, "size_j": sj,
                         "code_unit": code_unit, "speed": speed})
    constants = {k: getattr(vc, k) for k in ("ALPHA", "ASPR_0", "M_MOL", "REYNOLDS_0", "RHO_0", "SIGMA_0",
                                             "STOKES_0", "X_SEC")}
    return {"source": "val/swarm/src/validate_colphys.py local_pair_velocity", "constants": constants,
            "idx_p": 2.0, "idx_q": -1.0, "rows": rows}


def ref_host():
    from gamedev_b200 import workloads  # noqa: F401  (loads libgd_b200 for default configs)
    from oracle.ref import refhost

    out = {}
    rng = np.random.default_rng(77)
    for model in refhost.MODELS:
        h = refhost.RefHost(model)
        import oracle.ref.make_model as mm

        cfg = mm.model_config(model)
        y0, y1 = cfg.y_min, cfg.y_max
        pairs = []
        for _ in range(150):
            yi, yj = (float(rng.uniform(y0, 0.999 * y1)) for _ in range(2))
            zi = float(0.5 * math.pi + (rng.normal(0, 0.05) if cfg.n_z > 1 else 0.0))
            zj = float(0.5 * math.pi + (rng.normal(0, 0.05) if cfg.n_z > 1 else 0.0))
            smin, smax = max(cfg.init_smin, 1e-6), max(cfg.init_smax, cfg.init_smin * 10)
            si = float(math.exp(rng.uniform(math.log(smin), math.log(smax * 10))))
            sj = float(math.exp(rng.uniform(math.log(smin), math.log(smax * 10))))
            numr_j = float(10 ** rng.uniform(0, 20))
            lam = float(10 ** rng.uniform(-40, 0))
            meas = float(10 ** rng.uniform(20, 40)) if not cfg.code_unit else float(10 ** rng.uniform(-6, 0))
            r, v = h.pair_rate(yi, zi, yj, zj, si, sj, numr_j, lam, meas)
            pairs.append([yi, zi, yj, zj, si, sj, numr_j, lam, meas, r, v])
        moments = []
        for _ in range(200):
            si = float(math.exp(rng.uniform(math.log(cfg.init_smin), math.log(cfg.init_smin * 1e6))))
            q = float(10 ** rng.uniform(-9, 0.5))
            sj = si * q ** (1.0 / 3.0)
            high = int(rng.uniform() < 0.6)
            u = float(rng.uniform())
            f, m, s, x = h.outcome_moments(si, sj, high)
            moments.append([si, sj, high, u, f, m, s, x, h.sample_outcome(si, sj, high, u)])
        # near the monomer floor: the L < 1e-3 series branch of catastrophic fragmentation
        for _ in range(20):
            si = cfg.init_smin * (1.0 + float(rng.uniform(0, 2e-3)))
            sj = si * 0.9
            u = float(rng.uniform())
            f, m, s, x = h.outcome_moments(si, sj, 1)
            moments.append([si, sj, 1, u, f, m, s, x, h.sample_outcome(si, sj, 1, u)])
        measures = []
        for _ in range(150):
            y = float(rng.uniform(y0, 0.999 * y1))
            z = float(rng.uniform(cfg.z_min, cfg.z_max)) if cfg.n_z > 1 else 0.5 * math.pi
            r = float((y1 - y0) * 10 ** rng.uniform(-4, -0.3))
            measures.append([y, z, r, h.ball_measure(y, z, r)])
        out[model] = {"pair_rate": pairs, "moments": moments, "measure": measures}

    # controller scenarios with the reference's default bins (model "code": 8 x 4 x 2 groups)
    import oracle.ref.make_model as mm

    h = refhost.RefHost("code")
    cfg = mm.model_config("code")
    raw_count = h.lib.ref_raw_count()
    groups = raw_count // cfg.col_bin_s
    binmaps = []
    for _ in range(20):
        raw = rng.integers(0, 200, raw_count) * (rng.uniform(size=raw_count) < 0.6)
        merged, mp = h.binmap(raw)
        binmaps.append({"raw": raw.tolist(), "merged": merged, "map": mp.tolist()})
    chooses = []
    for _ in range(60):
        nb = int(rng.integers(1, 9))
        bins = np.zeros((nb, 6))
        bins[:, 0] = rng.uniform(0, 1, nb) * (rng.uniform(size=nb) < 0.8)
        bins[:, 1] = 10 ** rng.uniform(-3, 3, nb)
        bins[:, 2] = 10 ** rng.uniform(-4, 2, nb) * bins[:, 0]
        bins[:, 3] = 10 ** rng.uniform(-5, 1, nb) * bins[:, 0]
        bins[:, 4] = rng.integers(1, 500, nb)
        remaining = float(10 ** rng.uniform(-3, 1))
        scale = float(rng.choice([0.25, 0.5, 0.625, 1.0]))
        st, d, b = h.choose_bath(bins, remaining, scale)
        chooses.append({"bins": bins.tolist(), "remaining": remaining, "scale": scale, "status": st,
                        "duration": d, "binding": b})
    finishes = []
    for _ in range(60):
        nb = int(rng.integers(1, 9))
        a = np.zeros((nb, 15))
        mass = rng.uniform(0, 1, nb) * (rng.uniform(size=nb) < 0.9)
        a[:, 0] = mass
        p = rng.uniform(0, 1, nb)
        a[:, 1] = mass * p
        a[:, 2] = mass * p * rng.uniform(0.5, 2, nb)
        a[:, 3] = mass * mass * p * (1 - p) * 0.01
        a[:, 4] = mass * mass * p * 0.01
        a[:, 5] = mass * 10 ** rng.uniform(-4, -1, nb)
        a[:, 6] = mass * mass * 10 ** rng.uniform(-6, -2, nb)
        a[:, 7] = mass * rng.uniform(0.001, 0.1, nb)
        a[:, 8] = mass * rng.uniform(0.0, 0.2, nb)
        a[:, 9] = mass * np.clip(p * rng.uniform(0.5, 1.5, nb), 0, 1)
        a[:, 10] = mass * p * rng.uniform(0.5, 1.5, nb)
        a[:, 11] = mass * 10 ** rng.uniform(-4, -1, nb)
        a[:, 12] = mass * rng.uniform(0.9, 1.1, nb)
        a[:, 13] = rng.integers(1, 300, nb)
        state = [float(rng.choice([0.25, 0.5, 1.0])), int(rng.integers(0, 2)), int(rng.integers(0, 3)),
                 int(rng.integers(0, 2))]
        rc, st4, res = h.finish_bath(a, state)
        finishes.append({"audit": a.tolist(), "state": state, "status": rc, "state_out": st4.tolist(),
                         "result": res.tolist()})
    schedules = []
    for _ in range(6):
        G = groups
        W = (G + 31) // 32
        edges = np.zeros(G * W, np.uint32)
        for c in range(G):
            for d in range(G):
                if c == d or rng.uniform() < 0.08:
                    edges[c * W + d // 32] |= np.uint32(1 << (d % 32))
        horizon = float(10 ** rng.uniform(-2, 1))
        req = (horizon * 2.0 ** -rng.uniform(0, 7, G)).tolist()
        s = refhost.RefSchedule(h, horizon, req, edges)
        trace = {"edges": edges.tolist(), "horizon": horizon, "requested": req, "status": s.status, "steps": []}
        waves = 0
        while s.status == 0 and s.time() < s.end() and waves < 24:
            tick = s.time()
            due = s.due(tick)
            step = {"tick": tick, "due": due}
            if tick != 0:
                newreq = (horizon * 2.0 ** -rng.uniform(0, 7, G)).tolist()
                passed = (rng.uniform(size=G) < 0.7).astype(int).tolist()
                rc = s.adapt(tick, due, newreq, passed)
                step.update(requested=newreq, passed=passed, adapt_status=rc)
            step["levels"] = s.levels()
            s.advance(due)
            trace["steps"].append(step)
            waves += 1
        s.close()
        schedules.append(trace)
    out["controller"] = {"groups": groups, "bins": int(cfg.col_bin_s), "bin_min": int(cfg.col_bin_min),
                         "binmap": binmaps, "choose": chooses, "finish": finishes, "schedule": schedules}
    return out


if __name__ == "__main__":
    from oracle.ref import REFERENCE_ROOT

    reference = Path(sys.argv[1]) if len(sys.argv) > 1 else REFERENCE_ROOT
    (HERE / "colphys_golden.json").write_text(json.dumps(colphys(reference)))
    (HERE / "ref_host_golden.json").write_text(json.dumps(ref_host()))
    print("written", [p.name for p in HERE.glob("*.json")])
