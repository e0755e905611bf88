"""Time the reference's own CUDA collision step (oracle/_ref/collide_<model>_<n>/ref_collide) on a
benchmark workload, on this machine's GPU: geometry (site init, KD build, col_cache_get,
col_space_bin) plus two evolve_collisions half-operators, the swarm step bench.py times on the B200
path.  The half-operator length is set the same way: min(0.5/Omega(1 au), 2 / max bath-start rate),
the rates coming from one tiny operator of libgd_b200 on the same particles.  TEST INFRASTRUCTURE
ONLY: a reported reference figure, not part of the product.

    python oracle/ref/time_ref_collide.py [--workload c3_learned_3d] [--n 10000000]
"""

from __future__ import annotations

import argparse
import json
import math
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3_learned_3d")
    ap.add_argument("--n", type=int, default=None)
    a = ap.parse_args()

    import gamedev_b200 as gd
    from gamedev_b200 import workloads
    from oracle.ref import refcollide

    cfg = workloads.config(a.workload)
    n = a.n or workloads.CONFIGS[a.workload]["n"]
    p = workloads.particles(a.workload, n=n, seed=workloads.CONFIGS[a.workload]["seed"])
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(n, seed=1)
    sw.evolve_collisions(dp, rng, 1.0e-12 * workloads.orbital_time(), mass)
    rate_max = float(sw.owner_state()[0][:, 0].max().item())
    sw.close()
    del dp, rng
    half = min(0.5 * workloads.orbital_time(), 2.0 / rate_max)
    _, info = refcollide.run(a.workload, p, 1, half, mass, 2, timeout=3000)
    info.update(workload=a.workload, half_operator_s=half,
                steps_per_s=1e3 / info["total_ms"],
                impl="reference CUDA collision step (col_site_init + kdtree::buildTree + col_cache_get + "
                     "col_space_bin + 2 x evolve_local_collisions), sm_100a")
    print(json.dumps(info), flush=True)


if __name__ == "__main__":
    main()
