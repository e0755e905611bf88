#!/usr/bin/env python
"""Benchmark of the swarm collision hot path: exact kNN queries/s (and swarm steps/s) at N = 10^7,
K = 64 on synthetic data with the c3 shapes (3D disk, log-uniform radius, Gaussian vertical
profile, log-uniform grain radii).

The headline step is the learned-radius neighbour search, captured once as a CUDA graph and
replayed on drifted positions:

- geometry build: site init, Morton radix sort, bucket tree;
- radius features and the MLP's proposed radius;
- the radius-bounded exact top-K of every owner.

Twenty plain steps with Keplerian drift first train the MLP online. Every timed step is checked
bit-exact against the plain query. The line also reports:

- `plain`: the same search without the learned radius;
- `learned`: the eager, uncaptured learned step;
- `swarm_step`: geometry + top-K + two collision half-operators.

`value` is device-timed with inputs resident. `e2e` replays the same graph with the particles
copied in from pinned host memory, the deferred non-finite screen read, and codes and measure
copied back, all inside the timed region. `--impl reference` times the reference's own CUDA build
(compiled from the GameDev sources into oracle/_ref) on the same workload and GPU: its geometry
(site init, KD build, col_cache_get) as queries/s, and its swarm step; without that build it falls
back to the CPU restatement of the reference's KD search. Both arms report that CPU restatement as
`cpu_baseline`. Under torchrun every rank runs an independent replica (the path does not shard
across GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "exact kNN queries/s & swarm steps/s at N=1e7,K=64: learned-radius vs plain tree"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c3_learned_3d")
    ap.add_argument("--n", type=int, default=None, help="override the particle count (tests only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-step", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the C4 full Strang step line")
    ap.add_argument("--c4-n", type=int, default=None, help="C4 particle count (default: the workload's 1e7)")
    ap.add_argument("--c4-steps", type=int, default=2, help="timed C4 steps (the workload runs 1000)")
    ap.add_argument("--cpu-sample", type=int, default=200_000)
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi takes a few hundred ms to start: wait (bounded) for its first row so that the
        # samples cover the region that follows
        t_end = time.monotonic() + 5.0
        while time.monotonic() < t_end and self.proc.poll() is None:
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_init(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def _reduce_device():
    """Where a rank's scalar goes for a collective: host memory under gloo, the GPU under nccl."""
    import torch.distributed as dist

    return "cpu" if dist.get_backend() == "gloo" else "cuda"


def barrier(world):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def reduce_max(x, world):
    import torch

    if world <= 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, world):
    import torch

    if world <= 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def load_traffic(kernel: str, n: int, k: int):
    """dram bytes per launch of `kernel` from the committed ncu summary, scaled to n owners."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text()).get(kernel)
    if not d or d.get("k") != k:
        return None
    return d["dram_bytes_per_launch"] * n / d["n"]


def bench_config(workload, cfg, n, n_active, world):
    """The `config` of the JSON line; both arms print the same one for the same workload."""
    return {"workload": workload, "n": n, "k": cfg.n_k, "active": n_active,
            "geometry": "3d" if cfg.n_z > 1 else "2d",
            "step": "neighbour index build + exact top-K of every owner (codes and FP64 ball measure written)",
            "l2": "inputs and outputs larger than L2 (sites 16 B x N, codes 4K B x N)",
            "parallelism": f"replicas x{world}"}


def cpu_baseline(cfg, site4, q, active, sample, runs=5):
    """The oracle (the reference's KD tree and heap restated in C, OpenMP) on this machine's host
    cores: one KD build over all sites, then a bounded sample of owners queried; one warm-up run,
    then the median of `runs`, at all cores and at 1 thread (a tenth of the sample).  The value is
    the full step's throughput: active owners / (build time + the sample's query time scaled to all
    active owners)."""
    import numpy as np

    from oracle import oracle

    n = site4.shape[0]
    n_active = int(active.sum())
    cores = len(os.sched_getaffinity(0))
    t0 = time.perf_counter()
    tree = oracle.KdTree(site4, active)
    t_build = time.perf_counter() - t0
    # rows land at their owner's index; only the sampled rows' pages are ever touched
    codes = np.empty((n, cfg.n_k), np.int32)
    out = {}
    for label, threads, count in (("all", cores, min(sample, n)), ("one", 1, max(1, min(sample, n) // 10))):
        first = (n - count) // 2
        times = []
        for r in range(runs + 1):
            t0 = time.perf_counter()
            # rows land in the sample's own buffer (codes is indexed from `first`)
            tree.query(q, cfg.n_k, codes, None, threads=threads, first=first, count=count)
            if r:
                times.append(time.perf_counter() - t0)
        t_query = statistics.median(times)
        out[label] = {"threads": threads, "sample": count, "query_s": t_query,
                      "queries_per_s": n_active / (t_build + t_query * n_active / count)}
    tree.close()
    return {"value": out["all"]["queries_per_s"], "unit": "queries/s", "cores": cores, "kind": "port",
            "one_thread": out["one"]["queries_per_s"], "build_s": t_build, "runs": runs,
            "sample": (f"KD build over all {n} sites ({t_build:.2f} s, one thread) plus {out['all']['sample']} owners "
                       f"queried ({out['one']['sample']} at 1 thread), median of {runs} runs after one warm-up; value "
                       f"= active owners / (build + sample query time scaled to all active owners)")}


def run_reference(args):
    """--impl reference, rank 0 only.

    The reference's own CUDA build (oracle/_ref/collide_<workload>_<n>/ref_collide, compiled from
    the GameDev sources) on this machine's GPU, for the same workload: each step rebuilds the
    geometry (col_site_init, kdtree::buildTree, col_cache_get, col_space_bin) and runs two
    evolve_collisions half-operators.  `value` is active owners / the mean geometry time (the
    reference's exact kNN queries/s); swarm_step is its steps/s.  The CPU port of the same search is
    reported as cpu_baseline.  Where the reference build is absent, the CPU port is the value.
    Nothing here loads libgd_b200."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from gamedev_b200 import workloads
    from oracle import oracle
    from oracle.ref import refcollide

    cfg = workloads.config(args.workload)
    n = args.n or workloads.CONFIGS[args.workload]["n"]
    p = workloads.particles(args.workload, n=n, seed=workloads.CONFIGS[args.workload]["seed"])
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    site4, q, active, bad = oracle.site_init(cfg, p)
    if bad != -1:
        raise SystemExit(f"non-finite particle {bad}")
    n_active = int(active.sum())
    line = {"metric": METRIC, "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": bench_config(args.workload, cfg, n, n_active, world),
            "impl": "reference"}
    cb = cpu_baseline(cfg, site4, q, active, args.cpu_sample)
    half = workloads.swarm_half_operator(args.workload)
    have_gpu = subprocess.run(["nvidia-smi", "-L"], capture_output=True).returncode == 0 if _which("nvidia-smi") else False
    if refcollide.available(args.workload, n) and have_gpu:
        clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        _, info = refcollide.run(args.workload, p, 1, half, mass, operators=2, steps=args.warmup + args.steps,
                                 timeout=1800)
        clk = clocks.stop()
        timed = info["steps"][args.warmup:]
        geo_ms = statistics.mean(s[0] for s in timed)
        step_ms = statistics.mean(sum(s) for s in timed)
        value = n_active / (geo_ms / 1e3)
        line.update({
            "value": value, "ms_per_step": geo_ms,
            "reference_build": {"kind": "reference", "device": "cuda", "program": f"oracle/_ref/collide_{args.workload}_{n}/ref_collide",
                                "what": "GameDev's own CUDA sources (src/swarm/col_*.cu, kdtree/, _col_*.cuh) compiled for sm_100a; "
                                        "geometry = col_site_init + kdtree::buildTree + col_cache_get + col_space_bin",
                                "geometry_ms": geo_ms},
            "swarm_step": {"steps_per_s": 1e3 / step_ms, "ms_per_step": step_ms,
                           "definition": "geometry + 2 evolve_collisions half-operators of swarm_half_operator() "
                                         "seconds each (the same definition as the other arm)",
                           "half_operator_s": half},
            "clocks": clk,
        })
    else:
        line.update({"value": cb["value"], "ms_per_step": n_active / cb["value"] * 1e3,
                     "reference_build": {"kind": "port", "why": "the reference's CUDA build (oracle/_ref) or a GPU "
                                                                "is absent: the CPU port stands in"}})
    if not args.no_c4 and args.workload == "c3_learned_3d" and have_gpu:
        try:
            line["c4_step"] = c4_reference(args, args.c4_n or workloads.CONFIGS[C4]["n"], 1, max(1, args.c4_steps))
        except Exception as e:  # reported, never hidden
            line["c4_step"] = {"error": str(e)}
    line["cpu_baseline"] = cb
    line["e2e"] = {"value": line["value"], "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)


C4 = "c4_production_3d"
C4_DEFINITION = ("one Strang step of the c4 model (3D, N = 1e7, K = 64; drag and gravity, radiation pressure with "
                 "Poynting-Robertson drag, Ito diffusion, coagulation and fragmentation): dt = min(DT_MAX, 1/max rate, "
                 "dt_out - clock_out); C(dt/2) D(dt/2) T(dt) D(dt/2) C(dt/2), each C a geometry rebuild + exact top-K "
                 "+ frozen-bath collision operator")


def c4_step(args, gd, model, dev, world, rank, stream):
    """The C4 line: gd_step captured once into a CUDA graph (after two eager steps: buffers, then the
    learned search seeded by the first step's K-th distances) and replayed; device-timed."""
    import torch

    from gamedev_b200 import workloads

    n = args.c4_n or workloads.CONFIGS[C4]["n"]
    cfg = workloads.config(C4)
    run = workloads.run_info(C4)
    p = workloads.particles(C4, n=n, seed=workloads.CONFIGS[C4]["seed"] + rank)
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p, device=dev)
    rng = gd.rngstate_init(n, seed=4 + rank, device=dev)
    sw.set_clock(0.0, 0.0, run.dt_out)
    for _ in range(2):
        sw.step(run, dp, rng, mass, model)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sw.step(run, dp, rng, mass, model)
    graph.replay()
    sw.check_step()
    k = max(1, args.c4_steps)
    barrier(world)
    torch.cuda.nvtx.range_push("c4_step")
    a, b = _timed(stream, lambda: [graph.replay() for _ in range(k)])
    torch.cuda.nvtx.range_pop()
    barrier(world)
    ms = reduce_max(a.elapsed_time(b), world) / k
    sw.check_step()
    clk = sw.clock()
    ops = sw.last_operator_stats()
    del graph
    # one more step, eager, with COL_DIAGNOSTICS on (untimed): the operators' device-time split
    # between chains, audits and the rest (reservoir, bath rates, bins, controller) from their log
    sw.set_diagnostics(True)
    sw.step(run, dp, rng, mass, model)
    logged = sw.operator_log()[-2:]
    phases = sw.operator_phase_seconds()
    split = {"operators": len(logged), "seconds": phases,
             "waves": [e["waves"] for e in logged], "owner_updates": [e["owner_updates"] for e in logged],
             "events": [int(sum(e["event_counts"])) for e in logged]}
    sw.close()
    return {"steps_per_s": world * 1e3 / ms, "ms_per_step": ms, "n": n, "k": cfg.n_k, "steps_timed": k,
            "steps_before": 3, "dt_s": clk["dt"], "graph_captured": True, "learned_radius": True,
            "definition": C4_DEFINITION, "operators_of_timed_steps": ops, "operator_split": split,
            "note": "the workload runs 1000 such steps; a few are timed here; operator_split is one more "
                    "step with COL_DIAGNOSTICS on, device time"}


def c4_reference(args, n, warmup, steps):
    """The reference's C4 step on this GPU: its dynamics (oracle/_ref/step_c4_production_3d_<n>/ref_step:
    dyn_rate_calc + max_element, diffusion_pos, ssa_substep_1, optdepth_*, ssa_substep_2) plus two
    half-operators (oracle/_ref/collide_c4_production_3d_<n>/ref_collide: geometry + evolve_collisions
    of dt/2 each, dt the reference's own first timestep)."""
    from gamedev_b200 import workloads
    from oracle.ref import refcollide, refstep

    if not (refcollide.available(C4, n) and refstep.available(C4, n)):
        return {"unavailable": f"oracle/_ref builds of {C4} at {n} are absent"}
    p = workloads.particles(C4, n=n, seed=workloads.CONFIGS[C4]["seed"])
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    _, _, dyn = refstep.run(C4, p, 4, warmup + steps, mass, timeout=1800)
    dyn_ms = statistics.mean(dyn["ms"][warmup:])
    half = 0.5 * dyn["dt"][0]
    _, info = refcollide.run(C4, p, 4, half, mass, operators=1, steps=2 * (warmup + steps), timeout=1800)
    halves = info["steps"][2 * warmup:]
    col_ms = 2.0 * statistics.mean(sum(h) for h in halves)
    ms = dyn_ms + col_ms
    return {"steps_per_s": 1e3 / ms, "ms_per_step": ms, "n": n, "steps_timed": steps, "dt_s": dyn["dt"][0],
            "dynamics_ms": dyn_ms, "collision_halves_ms": col_ms, "definition": C4_DEFINITION,
            "programs": [f"oracle/_ref/step_{C4}_{n}/ref_step", f"oracle/_ref/collide_{C4}_{n}/ref_collide"]}


def _which(name):
    import shutil

    return shutil.which(name)


def _timed(stream, fn):
    import torch

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    return a, b


def run_ours(args):
    import numpy as np
    import torch

    import gamedev_b200 as gd
    from gamedev_b200 import workloads

    world, rank, local = dist_init(args.gpus)
    cfg = workloads.config(args.workload)
    n = args.n or workloads.CONFIGS[args.workload]["n"]
    K = cfg.n_k
    p_host = workloads.particles(args.workload, n=n, seed=workloads.CONFIGS[args.workload]["seed"] + rank)
    mass = float((p_host[:, 7] * math.pi * p_host[:, 6] ** 3 / 6.0).sum())
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()

    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p_host, device=dev)
    codes = torch.empty((n, K), dtype=torch.int32, device=dev)
    codes_ref = torch.empty((n, K), dtype=torch.int32, device=dev)
    measure = torch.empty(n, dtype=torch.float64, device=dev)
    kth = torch.empty(n, dtype=torch.float32, device=dev)
    stats = torch.zeros(4, dtype=torch.int64, device=dev)

    # ---- plain tree: geometry + exact top-K, inputs resident -------------------------------
    # the autotuner picks the sort order, walk, prescan depth and block width on this input
    # (every setting gives the same exact lists; it checks that too)
    plain_tuning, _ = sw.autotune(dp)
    for _ in range(args.warmup):
        sw.col_site_init(dp)
        sw.col_cache_get(dp, codes, measure, kth)
    site4, q, active = sw.get_sites()
    n_active = int(active.sum().item())
    plain_ev = []
    barrier(world)
    torch.cuda.nvtx.range_push("plain_step")
    for s_ in range(args.steps):
        e0 = _timed(stream, lambda: sw.col_site_init(dp))
        e1 = _timed(stream, lambda: sw.col_cache_get(dp, codes, measure, kth))
        plain_ev.append((e0, e1))
    torch.cuda.nvtx.range_pop()
    barrier(world)
    plain_build = statistics.mean(e[0][0].elapsed_time(e[0][1]) for e in plain_ev)
    plain_knn = statistics.mean(e[1][0].elapsed_time(e[1][1]) for e in plain_ev)
    plain_ms = reduce_max(plain_build + plain_knn, world)
    sw.col_cache_get_bounded(dp, None, codes, None, None, stats)
    torch.cuda.synchronize()
    plain_offers = float(stats[2].item()) / max(1, n_active)

    # ---- learned radius: 20 plain steps with Keplerian drift train the network online -----
    model = gd.RadiusModel(cfg.R_0, seed=1 + rank)
    drift_dt = 0.02 * workloads.orbital_time()
    prev = kth.clone()
    train_loss = None
    feats = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    for _ in range(20):
        sw.drift_keplerian(dp, drift_dt)
        sw.col_site_init(dp)
        sw.col_cache_get(dp, codes, measure, kth)
        sw.radius_features(dp, prev, mass, out=feats)
        train_loss = model.train(feats, kth, iterations=100, batch=16384, lr=2e-3)
        # the non-learned proposal's margin: the 0.999 quantile of log(r_now / r_prev), the K-th
        # distance's change over one step, taken from the last training step
        grow = 0.5 * torch.log(kth.clamp_min(1e-30) / prev.clamp_min(1e-30))
        heur_margin = float(torch.kthvalue(grow.cpu(), max(1, int(0.999 * n))).values.item())
        prev.copy_(kth)
    margin = model.calibrate(feats, kth, 0.999)
    radius = torch.empty(n, dtype=torch.float32, device=dev)
    # the radius-bounded query tunes its walk for the proposed radii (same sort order)
    sw.col_site_init(dp)
    sw.radius_features(dp, prev, mass, out=feats)
    model.predict(feats, out=radius)
    learned_tuning, _ = sw.autotune(dp, radius, tune_sort=False)

    def learned_step():
        sw.col_site_init(dp)
        sw.radius_features(dp, prev, mass, out=feats)
        model.predict(feats, out=radius)
        sw.col_cache_get_bounded(dp, radius, codes, measure, kth, stats)

    learned_ev, exact_steps = [], 0
    fallbacks = offers = 0
    for s_ in range(args.warmup + args.steps):
        sw.drift_keplerian(dp, drift_dt)  # positions move between steps (outside the timed region)
        stats.zero_()
        if s_ >= args.warmup:
            torch.cuda.nvtx.range_push("learned_step_eager")
        ev = _timed(stream, learned_step)
        if s_ >= args.warmup:
            torch.cuda.nvtx.range_pop()
            learned_ev.append(ev)
            # verification against the plain query on the same geometry (untimed)
            sw.col_cache_get(dp, codes_ref, None, None)
            exact_steps += int(torch.equal(codes, codes_ref))
            fallbacks += int(stats[3].item())
            offers += int(stats[2].item())
        prev.copy_(kth)
    barrier(world)
    learned_ms = reduce_max(statistics.mean(e[0].elapsed_time(e[1]) for e in learned_ev), world)
    queries = reduce_sum(float(n_active), world)
    learned_value = queries / (learned_ms / 1e3)
    plain_value = queries / (plain_ms / 1e3)

    # ---- ablation: what the network gains over the method without it ---------------------------
    # The same radius-bounded query, on the same fresh step, seeded either by the network or by the
    # previous step's K-th distance alone, r = sqrt(prev K-th d^2) * exp(m) with m calibrated like
    # the network's margin (0.999 quantile of the one-step change).  Both must give the plain rows.
    sw.drift_keplerian(dp, drift_dt)
    sw.col_site_init(dp)
    sw.radius_features(dp, prev, mass, out=feats)
    model.predict(feats, out=radius)
    radius_h = torch.sqrt(prev) * math.exp(heur_margin)
    sw.col_cache_get(dp, codes_ref, None, kth)
    ablation = {}
    for label, r in (("learned", radius), ("previous_kth", radius_h), ("none", None)):
        st = torch.zeros(4, dtype=torch.int64, device=dev)
        sw.col_cache_get_bounded(dp, r, codes, None, None, st)
        exact = bool(torch.equal(codes, codes_ref))
        evs = [_timed(stream, lambda: sw.col_cache_get_bounded(dp, r, codes, None, None, None))
               for _ in range(max(3, args.steps // 4))]
        torch.cuda.synchronize()
        st = st.cpu().tolist()
        ablation[label] = {"knn_query_ms": statistics.mean(a.elapsed_time(b) for a, b in evs),
                           "leaf_groups_per_owner": st[0] / max(1, n_active), "nodes_per_owner": st[1] / max(1, n_active),
                           "offers_per_owner": st[2] / max(1, n_active), "fallback_fraction": st[3] / max(1, n_active),
                           "bit_exact": exact}
    ablation["previous_kth"]["margin_log"] = heur_margin
    ablation["learned_vs_previous_kth"] = (ablation["previous_kth"]["knn_query_ms"]
                                           / ablation["learned"]["knn_query_ms"])
    prev.copy_(kth)

    # ---- the learned step captured once as a CUDA graph and replayed (the headline) ---------
    # The non-finite screen is deferred to check_geometry() so the step enqueues without a host
    # synchronisation; each replay reads the drifted positions from the same device buffer.
    sw.set_deferred_checks(True)

    def graph_body():
        sw.col_site_init(dp)
        sw.radius_features(dp, prev, mass, out=feats)
        model.predict(feats, out=radius)
        sw.col_cache_get_bounded(dp, radius, codes, measure, kth, None)

    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        graph_body()
    stream.wait_stream(side)
    launches_g0 = sw.launch_count()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        graph_body()
    graph_launches = sw.launch_count() - launches_g0 + 1  # + the radius model's MLP kernel
    graph_ev, graph_exact = [], 0
    # clocks from the timed replays through one more window of at least 2 s of the same replays
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    for s_ in range(args.warmup + args.steps):
        sw.drift_keplerian(dp, drift_dt)  # outside the timed region
        if s_ >= args.warmup:
            torch.cuda.nvtx.range_push("learned_step")
        ev = _timed(stream, graph.replay)
        if s_ >= args.warmup:
            torch.cuda.nvtx.range_pop()
            graph_ev.append(ev)
            sw.check_geometry()  # the deferred screen; also marks the replayed geometry valid
            sw.col_cache_get(dp, codes_ref, None, None)  # the plain query judges every step (untimed)
            graph_exact += int(torch.equal(codes, codes_ref))
        prev.copy_(kth)
    barrier(world)
    graph_ms = reduce_max(statistics.mean(e[0].elapsed_time(e[1]) for e in graph_ev), world)
    value = queries / (graph_ms / 1e3)

    # dominant kernel of the learned step (the bounded top-K), timed alone for the roofline
    knn_alone = []
    for _ in range(args.steps):
        knn_alone.append(_timed(stream, lambda: sw.col_cache_get_bounded(dp, radius, codes, measure, kth, None)))
    barrier(world)
    t_end = time.monotonic() + 2.0
    done = 0
    while done < args.steps or time.monotonic() < t_end:
        sw.drift_keplerian(dp, drift_dt)
        graph.replay()
        done += 1
        if done % 8 == 0:
            stream.synchronize()
    stream.synchronize()
    barrier(world)
    clk = clocks.stop()
    sw.check_geometry()
    launches = graph_launches
    knn_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in knn_alone)

    peak, peak_kind = peaks()
    bytes_per_query = 24 + 4 * K
    achieved = n_active * bytes_per_query / (knn_ms / 1e3) / 1e9
    traffic = load_traffic("k_knn_range", n_active, K)

    result = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": graph_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(args.workload, cfg, n, n_active, world),
        "impl_detail": {"index": "Morton bucket tree, 32-site buckets", "order": "ascending (d2, code)",
                        "step": "geometry build + features + MLP + radius-bounded top-K, one CUDA graph replay"},
        "plain": {"queries_per_s": plain_value, "ms_per_step": plain_ms, "geometry_build_ms": plain_build,
                  "knn_query_ms": plain_knn, "offers_per_owner": plain_offers, "tuning": plain_tuning},
        "graph": {"queries_per_s": value, "vs_plain": value / plain_value, "ms_per_step": graph_ms,
                  "bit_exact_steps": f"{graph_exact}/{args.steps}", "kernels_per_step": graph_launches,
                  "tuning": learned_tuning},
        "learned": {"queries_per_s": learned_value, "vs_plain": learned_value / plain_value, "ms_per_step": learned_ms,
                    "knn_query_ms": knn_ms, "hit_rate": 1.0 - fallbacks / max(1, n_active * args.steps),
                    "fallback_fraction": fallbacks / max(1, n_active * args.steps),
                    "offers_per_owner": offers / max(1, n_active * args.steps),
                    "bit_exact_steps": f"{exact_steps}/{args.steps}", "margin_log": margin,
                    "train_loss": train_loss, "training": "20 plain steps, 100 Adam iterations each, batch 16384",
                    "drift_between_steps": "Keplerian, 0.02/Omega(1 au)"},
        "ablation": ablation,
        "roofline": {"bound": "hbm", "kernel": "k_knn_range (the radius-bounded top-K call: range query + "
                                               "heap fallback for leftover owners)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "bytes_per_unit": bytes_per_query, "units_per_launch": n_active, "traffic": traffic},
        "clocks": clk,
        "gpu_launches": launches,
    }
    if exact_steps != args.steps or graph_exact != args.steps:
        result["error"] = "learned-radius neighbour lists differ from the plain query"

    # ---- end to end through the C ABI with host buffers (learned path) ---------------------
    # Each step copies its particles in from pinned host memory, replays the captured learned
    # step, reads the deferred non-finite screen and copies codes and measure back.  Inputs and
    # outputs are double-buffered (a second graph reads and writes the other pair): step k+1's
    # particles stream in on one copy stream and step k's results stream out on another while
    # the device computes, as a host that keeps the device busy would.
    if not args.no_e2e:
        p_now = dp.cpu()
        host_in = p_now.pin_memory()
        dp_b = [dp, torch.empty_like(dp)]
        codes_b = [codes, torch.empty_like(codes)]
        measure_b = [measure, torch.empty_like(measure)]
        dp_b[1].copy_(dp)
        graphs = [graph]

        def body1():
            sw.col_site_init(dp_b[1])
            sw.radius_features(dp_b[1], prev, mass, out=feats)
            model.predict(feats, out=radius)
            sw.col_cache_get_bounded(dp_b[1], radius, codes_b[1], measure_b[1], kth, None)

        side.wait_stream(stream)
        with torch.cuda.stream(side):
            body1()
        stream.wait_stream(side)
        g2 = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g2):
            body1()
        graphs.append(g2)
        host_codes = [torch.empty((n, K), dtype=torch.int32).pin_memory() for _ in range(2)]
        host_measure = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
        # results leave on two copy streams (two copy engines), each with half of the codes
        h2d_stream = torch.cuda.Stream()
        d2h_streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        h2d_done = [torch.cuda.Event(), torch.cuda.Event()]
        d2h_done = [[torch.cuda.Event(), torch.cuda.Event()] for _ in range(2)]
        computed = [torch.cuda.Event(), torch.cuda.Event()]
        half = n // 2

        def prefetch(t):
            b = t % 2
            h2d_stream.wait_event(computed[b])  # the step two back has finished reading buffer b
            with torch.cuda.stream(h2d_stream):
                dp_b[b].copy_(host_in, non_blocking=True)
            h2d_done[b].record(h2d_stream)

        def e2e_steps(count):
            prefetch(0)
            for t in range(count):
                b = t % 2
                if t + 1 < count:
                    prefetch(t + 1)
                stream.wait_event(h2d_done[b])  # this step's particles are in
                for ev in d2h_done[b]:
                    stream.wait_event(ev)  # buffer b's results (two steps back) are out
                graphs[b].replay()
                computed[b].record(stream)
                sw.check_geometry()  # the deferred non-finite screen of this step's input
                for h, st in enumerate(d2h_streams):
                    st.wait_event(computed[b])
                    lo, hi = (0, half) if h == 0 else (half, n)
                    with torch.cuda.stream(st):
                        host_codes[b][lo:hi].copy_(codes_b[b][lo:hi], non_blocking=True)
                        if h == 1:
                            host_measure[b].copy_(measure_b[b], non_blocking=True)
                    d2h_done[b][h].record(st)
            for st in d2h_streams:
                stream.wait_stream(st)  # the timed region ends after the last copy back

        e2e_steps(max(2, args.warmup))
        barrier(world)
        a, b = _timed(stream, lambda: e2e_steps(args.steps))
        barrier(world)
        e_ms = reduce_max(a.elapsed_time(b), world)
        result["e2e"] = {"value": queries * args.steps / (e_ms / 1e3), "unit": "queries/s",
                         "h2d_bytes_per_step": n * 64, "d2h_bytes_per_step": n * K * 4 + n * 8,
                         "ms_per_step": e_ms / args.steps,
                         "overlap": "inputs and outputs double-buffered: step k+1's particles in on one copy "
                                    "stream and step k's results out on two while the device computes; bound by "
                                    "the host link (2.64 GB out per step)"}
        del host_in, host_codes, host_measure, graphs, g2, codes_b, measure_b, dp_b

    del graph
    sw.set_deferred_checks(False)

    # ---- swarm step: geometry + top-K + two collision half-operators (learned and plain) ------
    if not args.no_step:
        try:
            # the particles as the learned steps left them (drifted positions, initial sizes); the
            # half-operator length is the workload's fixed one (the reference arm uses the same)
            half = workloads.swarm_half_operator(args.workload)
            sw.invalidate_col_geometry()
            rng = gd.rngstate_init(n, seed=1 + rank, device=dev)
            sw.evolve_collisions(dp, rng, 1.0e-12 * workloads.orbital_time(), mass)
            rate_max = float(sw.owner_state()[0][:, 0].max().item())
            rng = gd.rngstate_init(n, seed=1 + rank, device=dev)

            def swarm_step():
                sw.invalidate_col_geometry()
                sw.evolve_collisions(dp, rng, half, mass)
                sw.evolve_collisions(dp, rng, half, mass)

            kth_s = torch.empty(n, dtype=torch.float32, device=dev)

            def swarm_step_learned():
                # the learned-radius neighbour search fills the handle's cache, which both
                # half-operators then use (geometry and cache valid: no second search)
                sw.col_site_init(dp)
                sw.radius_features(dp, prev, mass, out=feats)
                model.predict(feats, out=radius)
                sw.col_cache_get_bounded(dp, radius, None, None, kth_s)
                prev.copy_(kth_s)
                sw.evolve_collisions(dp, rng, half, mass)
                sw.evolve_collisions(dp, rng, half, mass)

            st_steps = max(1, min(args.steps, 3))
            timings = {}
            for label, fn in (("plain", swarm_step), ("learned", swarm_step_learned)):
                fn()
                barrier(world)
                torch.cuda.nvtx.range_push(f"swarm_step_{label}")
                a, b = _timed(stream, lambda: [fn() for _ in range(st_steps)])
                torch.cuda.nvtx.range_pop()
                barrier(world)
                timings[label] = reduce_max(a.elapsed_time(b), world) / st_steps
            last_operator = sw.last_operator_stats()

            # The same learned step captured once as a CUDA graph: the search with its screen
            # deferred, and two operators whose waves run as conditional WHILE nodes with the
            # controller on the device.  From one saved state (particles, RNG, previous K-th
            # distances, bath controller reset), the replays must equal eager steps bit for bit.
            def swarm_step_ops():
                sw.col_site_init(dp)
                sw.radius_features(dp, prev, mass, out=feats)
                model.predict(feats, out=radius)
                sw.col_cache_get_bounded(dp, radius, None, None, kth_s)
                prev.copy_(kth_s)
                sw.evolve_local_collisions(dp, rng, half, mass)
                sw.evolve_local_collisions(dp, rng, half, mass)

            saved = (dp.clone(), rng.clone(), prev.clone())

            def restore():
                dp.copy_(saved[0])
                rng.copy_(saved[1])
                prev.copy_(saved[2])
                sw.reset_controller()

            sw.set_deferred_checks(True)
            restore()
            swarm_step_ops()  # eager warm-up: kernel attributes, operator scratch
            sw.check_geometry()
            step_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(step_graph):
                swarm_step_ops()
            restore()
            barrier(world)
            torch.cuda.nvtx.range_push("swarm_step_graph")
            a, b = _timed(stream, lambda: [step_graph.replay() for _ in range(st_steps)])
            torch.cuda.nvtx.range_pop()
            barrier(world)
            g_ms = reduce_max(a.elapsed_time(b), world) / st_steps
            sw.check_geometry()
            sw.check_operator()
            captured = dp.clone()
            restore()
            for _ in range(st_steps):
                swarm_step_ops()
            sw.check_geometry()
            torch.cuda.synchronize()
            graph_exact = bool(torch.equal(captured.view(torch.int64), dp.view(torch.int64)))
            sw.set_deferred_checks(False)
            del step_graph, captured, saved

            s_ms = min(timings["learned"], g_ms) if graph_exact else timings["learned"]
            result["swarm_step"] = {"steps_per_s": world * 1e3 / s_ms, "ms_per_step": s_ms,
                                    "graph_captured": graph_exact and g_ms <= timings["learned"],
                                    "graph": {"ms_per_step": g_ms, "steps_per_s": world * 1e3 / g_ms,
                                              "bit_exact_vs_eager": graph_exact, "steps": st_steps},
                                    "eager_learned_ms_per_step": timings["learned"],
                                    "plain_steps_per_s": world * 1e3 / timings["plain"],
                                    "plain_ms_per_step": timings["plain"],
                                    "definition": "geometry + exact top-K (learned radius; plain: without) + 2 "
                                                  "collision half-operators of swarm_half_operator() seconds each",
                                    "half_operator_s": half, "max_bath_rate_per_s": rate_max,
                                    "expected_events_fastest_owner": half * rate_max,
                                    "last_operator": last_operator}
        except Exception as e:  # reported, never hidden
            result["swarm_step"] = {"error": str(e)}

    # ---- C4: the full Strang step C(dt/2) D(dt/2) T(dt) D(dt/2) C(dt/2), one captured graph ----
    if not args.no_c4 and args.workload == "c3_learned_3d":
        try:
            result["c4_step"] = c4_step(args, gd, model, dev, world, rank, stream)
        except Exception as e:  # reported, never hidden
            result["c4_step"] = {"error": str(e)}

    # ---- CPU baseline: the oracle on the host cores, rank 0 at N = 1 -----------------------
    if not args.no_cpu and rank == 0 and world == 1:
        from oracle import oracle

        site4_h, q_h, active_h, _ = oracle.site_init(cfg, p_host)
        result["cpu_baseline"] = cpu_baseline(cfg, site4_h, q_h, active_h, args.cpu_sample)
    if rank == 0:
        print(json.dumps(result), flush=True)
    model.close()
    sw.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_batched(args):
    """The batched configuration (256 c0-shaped swarms, log-uniform sizes on [2^10, 2^18], K from
    {16, 32, 64}): segmented geometry + one persistent top-K launch, captured as one CUDA graph,
    against the same swarms searched one handle at a time.  Every swarm is checked bit-exact
    against its one-swarm result."""
    import torch

    import gamedev_b200 as gd
    from gamedev_b200 import workloads

    world, rank, local = dist_init(args.gpus)
    cfg, sizes, ks, p = workloads.c2_batch(seed=5 + rank)
    stream = torch.cuda.current_stream()
    dp = gd.particles_to_device(p)
    batch = gd.SwarmBatch(cfg, sizes, ks)
    # the key length the single-swarm autotuner picks at c3: the top 16 Morton bits per dimension
    # (6 radix passes in 3D instead of 8); the rows are exact for any key order
    sort_bits = 16 * (3 if cfg.n_z > 1 else 2)
    batch.set_tuning(sort_bits=sort_bits)
    codes, measure, kth = batch.outputs()
    side = torch.cuda.Stream()
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        for _ in range(args.warmup):
            batch.knn(dp, codes, measure, kth)
    stream.wait_stream(side)
    batch.check()
    graph = torch.cuda.CUDAGraph()
    l0 = batch.launch_count()
    with torch.cuda.graph(graph):
        batch.knn(dp, codes, measure, kth)
    kernels = batch.launch_count() - l0
    for _ in range(args.warmup):
        graph.replay()
    barrier(world)
    # clocks over the timed replays and at least 2 s of the same replays after them
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    t_end = time.monotonic() + 2.0
    torch.cuda.nvtx.range_push("c2_step")
    a, b = _timed(stream, lambda: [graph.replay() for _ in range(args.steps)])
    torch.cuda.nvtx.range_pop()
    while time.monotonic() < t_end:
        graph.replay()
        stream.synchronize()
    barrier(world)
    clk = clocks.stop()
    batch.check()
    b_ms = reduce_max(a.elapsed_time(b) / args.steps, world)
    # the same swarms one handle at a time (geometry + top-K per swarm, eager)
    solos = []
    for s_, n_s in enumerate(sizes):
        c = workloads.config("c0_plain_small", k=ks[s_])
        sw = gd.SwarmCollision(c, n_s)
        sl = dp[int(batch.part_off[s_]):int(batch.part_off[s_ + 1])]
        out = (torch.empty((n_s, ks[s_]), dtype=torch.int32, device=dp.device),
               torch.empty(n_s, dtype=torch.float64, device=dp.device),
               torch.empty(n_s, dtype=torch.float32, device=dp.device))
        solos.append((sw, sl, out))
    for sw, sl, out in solos:
        sw.col_site_init(sl)
        sw.col_cache_get(sl, *out)
    barrier(world)
    a, b = _timed(stream, lambda: [(sw.col_site_init(sl), sw.col_cache_get(sl, *out)) for sw, sl, out in solos])
    barrier(world)
    solo_ms = reduce_max(a.elapsed_time(b), world)
    exact = 0
    for s_, (sw, sl, out) in enumerate(solos):
        exact += int(torch.equal(batch.codes_of(codes, s_), out[0])
                     and torch.equal(batch.rows_of(measure, s_).view(torch.int64), out[1].view(torch.int64))
                     and torch.equal(batch.rows_of(kth, s_).view(torch.int32), out[2].view(torch.int32)))
    del graph

    # ---- the full collision step of every swarm: search + operator, one graph --------------
    # Each swarm's operator length gives its fastest owner ~10 expected events at bath start (the
    # solo handles measure the rates); the step (segmented geometry, persistent top-K, every
    # swarm's operator graph side by side) is captured once and replayed.  A sample of swarms is
    # checked against solo operators from the same state, bit for bit.
    collide = {}
    try:
        masses, durations = [], []
        for s_, (sw, sl, out) in enumerate(solos):
            pm = p[int(batch.part_off[s_]):int(batch.part_off[s_ + 1])]
            masses.append(float((pm[:, 7] * math.pi * pm[:, 6] ** 3 / 6.0).sum()))
            probe = sl.clone()
            sw.evolve_collisions(probe, gd.rngstate_init(sizes[s_], seed=3, device=dp.device),
                                 1.0e-12 * workloads.orbital_time(), masses[-1])
            durations.append(10.0 / max(float(sw.owner_state()[0][:, 0].max().item()), 1e-300))
        rng0 = torch.cat([gd.rngstate_init(n_s, seed=100 * rank + s_, device=dp.device) for s_, n_s in enumerate(sizes)])
        dp0 = dp.clone()
        rng = rng0.clone()
        batch.knn(dp, codes, measure, kth)
        batch.check()
        batch.collide(dp, rng, codes, measure, durations, masses)  # eager: the first operator of each swarm
        first = dp.clone()
        stats = [batch.operator_stats(s_) for s_ in range(len(sizes))]
        # solo operators of a sample of swarms from the same state, with fresh controllers
        sample = list(range(0, len(sizes), max(1, len(sizes) // 16)))
        same = 0
        for s_ in sample:
            sw, sl, out = solos[s_]
            lo, hi = int(batch.part_off[s_]), int(batch.part_off[s_ + 1])
            part_s = dp0[lo:hi].clone()
            rng_s = rng0.view(-1, gd.rng_state_bytes())[lo:hi].clone().view(-1)
            sw.reset_controller()
            sw.invalidate_col_geometry()
            sw.evolve_collisions(part_s, rng_s, durations[s_], masses[s_])
            same += int(torch.equal(first[lo:hi].view(torch.int64), part_s.view(torch.int64)))
        dp.copy_(dp0)
        rng.copy_(rng0)
        batch.reset_controller()
        step_graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(step_graph):
            batch.knn(dp, codes, measure, kth)
            batch.collide(dp, rng, codes, measure, durations, masses)
        step_graph.replay()
        batch.check()
        # every timed replay starts from the same state (particles, RNG, fresh controllers): the
        # operators grow the grains, and later steps of a run would hold ever more events
        times = []
        for _ in range(args.steps):
            dp.copy_(dp0)
            rng.copy_(rng0)
            batch.reset_controller()
            barrier(world)
            a, b = _timed(stream, step_graph.replay)
            barrier(world)
            times.append(reduce_max(a.elapsed_time(b), world))
        c_ms = statistics.mean(times)
        batch.check()
        collide = {"steps_per_s": world * 1e3 / c_ms, "ms_per_step": c_ms,
                   "definition": "segmented geometry + exact top-K + every swarm's frozen-bath collision operator "
                                 "(each ~10 expected events for its fastest owner), one CUDA graph replay, every "
                                 "timed replay from the same initial state",
                   "bit_exact_swarms_sampled": f"{same}/{len(sample)}",
                   "waves_per_swarm_max": max(st["waves"] for st in stats),
                   "events_total": int(sum(st["events"] for st in stats))}
        del step_graph
    except Exception as e:  # reported, never hidden
        collide = {"error": str(e)}
    for sw, sl, out in solos:
        sw.close()
    queries = reduce_sum(float(sum(sizes)), world)
    line = {
        "metric": "exact kNN queries/s, batched swarms", "value": queries / (b_ms / 1e3), "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": b_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "c2_batched", "swarms": len(sizes), "particles": int(sum(sizes)),
                   "n_range": [min(sizes), max(sizes)], "k_choices": [16, 32, 64],
                   "step": "segmented geometry (one launch per stage for all swarms) + one persistent top-K launch, one CUDA graph replay",
                   "sort_bits": sort_bits,
                   "parallelism": f"replicas x{world}"},
        "kernels_per_step": kernels,
        "one_handle_at_a_time": {"ms_per_step": solo_ms, "queries_per_s": queries / (solo_ms / 1e3)},
        "speedup_vs_one_at_a_time": solo_ms / b_ms,
        "bit_exact_swarms": f"{exact}/{len(sizes)}",
        "collision_step": collide,
        "clocks": clk,
    }
    if exact != len(sizes):
        line["error"] = "batched rows differ from the one-swarm results"
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_rates(args):
    """The FP64 bath-rate kernel alone (gd_bath_rates: col_bath_rate for every owner) on the c4
    shapes: every owner's K pair rates, outcome moments and fold, timed with CUDA events.  A line
    for the kernel that holds half of the C4 operator; also the command its ncu capture profiles
    (the operator's own launches sit inside a conditional graph, which ncu does not list)."""
    import torch

    import gamedev_b200 as gd
    from gamedev_b200 import workloads

    world, rank, local = dist_init(args.gpus)
    n = args.n or workloads.CONFIGS[C4]["n"]
    cfg = workloads.config(C4)
    p = workloads.particles(C4, n=n, seed=workloads.CONFIGS[C4]["seed"] + rank)
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p)
    sw.build_cache(dp)
    out = torch.empty((n, 4), dtype=torch.float64, device=dp.device)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        sw.bath_rates(dp, mass, out)
    barrier(world)
    evs = [_timed(stream, lambda: sw.bath_rates(dp, mass, out)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    ms = reduce_max(statistics.mean(a.elapsed_time(b) for a, b in evs), world)
    pairs = reduce_sum(float(n) * cfg.n_k, world)
    if rank == 0:
        print(json.dumps({"metric": "bath-start pair rates/s (col_bath_rate alone)", "value": pairs / (ms / 1e3),
                          "unit": "pair rates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic",
                          "config": {"workload": "c4_rates", "n": n, "k": cfg.n_k,
                                     "step": "env cache + disk heights + every owner's K pair rates and moments"}}),
              flush=True)
    sw.close()


def run_chain(args):
    """One frozen bath of the event chain for every owner (gd_bath_chain: bath-start rates, skip scan
    and chain, launched eagerly) on the c4 shapes, with the bath of the C4 operator's finest level
    (dt/2 over 32 waves, 3383 s).  Every timed call starts from the same particles and RNG streams.
    The command the chain kernel's ncu capture profiles: inside the operator it runs in a
    conditional graph, which ncu does not list."""
    import torch

    import gamedev_b200 as gd
    from gamedev_b200 import workloads

    world, rank, local = dist_init(args.gpus)
    n = args.n or workloads.CONFIGS[C4]["n"]
    cfg = workloads.config(C4)
    p = workloads.particles(C4, n=n, seed=workloads.CONFIGS[C4]["seed"] + rank)
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    bath = 3383.0
    sw = gd.SwarmCollision(cfg, n)
    dp0 = gd.particles_to_device(p)
    sw.build_cache(dp0)
    rng0 = gd.rngstate_init(n, seed=4 + rank)
    dp, rng = dp0.clone(), rng0.clone()
    stream = torch.cuda.current_stream()
    counts = []

    def one():
        counts.append(sw.bath_chain(dp, rng, mass, bath))

    for _ in range(args.warmup):
        dp.copy_(dp0)
        rng.copy_(rng0)
        one()
    barrier(world)
    evs = []
    for _ in range(args.steps):
        dp.copy_(dp0)
        rng.copy_(rng0)
        evs.append(_timed(stream, one))
    torch.cuda.synchronize()
    ms = reduce_max(statistics.mean(a.elapsed_time(b) for a, b in evs), world)
    events = reduce_sum(float(counts[-1]), world)
    if rank == 0:
        print(json.dumps({"metric": "events/s of one frozen bath (col_bath_rate + col_skip_scan + col_chain_run)",
                          "value": events / (ms / 1e3), "unit": "events/s", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": "c4_chain", "n": n, "k": cfg.n_k, "bath_s": bath,
                                     "events_per_step": counts[-1], "same_events_every_step": len(set(counts)) == 1,
                                     "step": "env cache + every owner's bath-start rates + skip scan + chain"}}),
              flush=True)
    sw.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload in ("c4_rates", "c4_chain"):
        import gamedev_b200

        gamedev_b200.load()
        (run_rates if args.workload == "c4_rates" else run_chain)(args)
        return
    if args.workload == "c2_batched":
        import gamedev_b200

        gamedev_b200.load()
        run_batched(args)
        return
    import gamedev_b200

    gamedev_b200.load()  # the prebuilt in-tree libgd_b200.so; raises if it is missing
    run_ours(args)


if __name__ == "__main__":
    main()
