"""Time the reference's own CUDA KD search (oracle/_ref/ref_knn) on a benchmark workload, on this
machine's GPU: KD build (kdtree::buildTree) and the col_cache_get-style top-K query, mean of
`--repeats` launches after one untimed launch, no neighbour output written (as the reference's KNN
harness times its queries).  TEST INFRASTRUCTURE ONLY: a reported reference figure, not part of
the product.

    python oracle/ref/time_ref_knn.py [--workload c3_learned_3d] [--n 10000000] [--repeats 3]
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3_learned_3d")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--repeats", type=int, default=3)
    a = ap.parse_args()

    from gamedev_b200 import workloads
    from oracle import oracle
    from oracle.ref import refknn

    cfg = workloads.config(a.workload)
    n = a.n or workloads.CONFIGS[a.workload]["n"]
    p = workloads.particles(a.workload, n=n, seed=workloads.CONFIGS[a.workload]["seed"])
    site4, q, active, bad = oracle.site_init(cfg, p)
    if bad != -1:
        raise SystemExit(f"non-finite particle {bad}")
    _, _, info = refknn.run(site4, q, active, cfg.n_k, repeats=a.repeats, outputs=False, timeout=3000)
    info.update(workload=a.workload, queries_per_s=info["queries"] / (info["query_ms"] / 1e3),
                impl="reference CUDA KD search (kdtree::buildTree + idx_old_heap + cct::knn), sm_100a")
    print(json.dumps(info), flush=True)


if __name__ == "__main__":
    main()
