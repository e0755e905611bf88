"""The B200 neighbour search against the reference's own CUDA KD search on the same GPU.

oracle/_ref/ref_knn compiles the reference's KD builder, index heap and traversal from the GameDev
tree (oracle/ref/Makefile) and drives them as col_cache_get does.  Both searches get the same sites
(the device's own site-init output).  Bar: every row's codes identical after the reference's heap
order is sorted to ascending (d^2, code) (its neighbour set and distances bit-exact), and the kept
K-th d^2 bit-identical.  Cases: the labelled edge cases and the c0 / c1 / c3 shapes.
"""

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu


def _ref():
    from oracle.ref import refknn

    if not refknn.available():
        pytest.skip("oracle/_ref/ref_knn was not built (the reference tree was absent at build time)")
    return refknn


def _compare(gd, cfg, p, name):
    import torch

    refknn = _ref()
    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    codes, measure, kth = sw.knn(dp)
    site4, q, active = (t.cpu().numpy() for t in sw.get_sites())
    torch.cuda.synchronize()
    codes, kth = codes.cpu().numpy(), kth.cpu().numpy()
    sw.close()
    rc, rd2, _ = refknn.run(site4, q, active, cfg.n_k)
    rc, rd2, rkth = refknn.canonical(rc, rd2)
    bad = np.nonzero((rc != codes).any(axis=1))[0]
    assert bad.size == 0, (name, int(bad.size), int(bad[0]), rc[bad[0]][:8], codes[bad[0]][:8])
    act = active.astype(bool)
    assert np.array_equal(rkth[act].view(np.uint32), kth[act].view(np.uint32)), name


@pytest.mark.parametrize("idx", range(11))
def test_edge_cases_match_reference_cuda(gd, cuda, idx):
    name, cfg, p = cases.small_cases(gd)[idx]
    _compare(gd, cfg, p, name)


@pytest.mark.parametrize("workload,n", [("c0_plain_small", 65536), ("c1_multisize_2d", 1 << 18),
                                        ("c3_learned_3d", 1 << 18)])
def test_workloads_match_reference_cuda(gd, cuda, workload, n):
    from gamedev_b200 import workloads

    _compare(gd, workloads.config(workload), workloads.particles(workload, n=n), workload)
