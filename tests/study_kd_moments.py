"""The KD-search moment study against the reference's CUDA build: a long GPU study (about 12
minutes), outside the regular suites because of its length.  Run it by naming the file:

    python -m pytest tests/study_kd_moments.py -q -s

The regular statistical parity test (16 seeds, ~10 events for the fastest owner) is
tests/test_ref_gpu_collide.py::test_kd_operator_matches_reference_cuda_statistically.
"""

import numpy as np
import pytest

from tests.test_ref_gpu_collide import N, _bootstrap_ratio, _duration, _mass, _moment, _ours, _refc

pytestmark = pytest.mark.gpu


def test_kd_moments_over_longer_operator_with_bootstrap(gd, cuda):
    """A study (about 12 minutes, most of it the reference's runs): the KD moments
    over an operator of ~100 expected events for the fastest owner, 16 seeds on each side, against
    the reference's CUDA build (c0 shapes, coagulation only).  M_0 agrees within 1% and M_1 (the dust
    mass) to 1e-12.  For M_2 it prints the ratio of the pooled means with a 95% bootstrap interval
    over seeds, beside the same interval for the reference against itself (seeds 1-8 against
    9-16), and the reference's per-seed spread.  Runaway growth from monodisperse grains makes the
    per-seed M_2 heavy-tailed: the reference's own self-interval spans tens of per cent, so a 1% bar
    on M_2 cannot be resolved with 16 seeds (a standard error of 1% would take about
    (spread / 0.01)^2 seeds per side).  The M_2 samples must agree by rank (Mann-Whitney, p > 0.01)."""
    from scipy.stats import mannwhitneyu

    from gamedev_b200 import workloads

    refcollide = _refc()
    model = "c0_plain_small"
    if not refcollide.available(model, N):
        pytest.fail("oracle/_ref reference collision build absent: build the checker first")
    cfg = workloads.config(model)
    p = workloads.particles(model, n=N, seed=12)
    d = _duration(gd, cfg, p, 100.0)
    mo = [[], [], []]
    mr = [[], [], []]
    for seed in range(1, 17):
        ours, _ = _ours(gd, cfg, p, seed, d)
        ref, _ = refcollide.run(model, p, seed, d, _mass(p), 1, timeout=900)
        for k in range(3):
            mo[k].append(_moment(ours, k))
            mr[k].append(_moment(ref, k))
    r0, lo0, hi0 = _bootstrap_ratio(mo[0], mr[0])
    r2, lo2, hi2 = _bootstrap_ratio(mo[2], mr[2])
    s2, slo2, shi2 = _bootstrap_ratio(mr[2][:8], mr[2][8:])
    spread = float(np.std(mr[2]) / np.mean(mr[2]))
    pval = float(mannwhitneyu(mo[2], mr[2]).pvalue)
    print(f"M0 ratio {r0:.5f} [{lo0:.5f}, {hi0:.5f}]; M2 ratio {r2:.4f} [{lo2:.4f}, {hi2:.4f}]; "
          f"reference M2 self-ratio {s2:.4f} [{slo2:.4f}, {shi2:.4f}]; reference per-seed M2 spread {spread:.3f}; "
          f"M2 Mann-Whitney p {pval:.3f}; seeds for a 1% standard error ~{(spread / 0.01) ** 2:.0f}")
    assert abs(r0 - 1.0) < 0.01, (r0, lo0, hi0)
    assert abs(np.mean(mo[1]) / np.mean(mr[1]) - 1.0) < 1e-12
    assert pval > 0.01, (pval, mo[2], mr[2])
    assert shi2 - slo2 > 0.02, (s2, slo2, shi2)  # the resolution 16 seeds give is coarser than 1%
