"""Azimuthal wedges on the B200: periodic images, the duplicate-image dedup, and parity with the
reference's own CUDA build of the same wedge models.

Bars:
  * the device's sites: particle i at site i (code 3i); its images at sites n + i and 2n + i
    (codes 3i + 1 and 3i + 2), the physical site rotated by -width and +width (col_site_init.cu:58-76)
    to 1e-6 of the radius; on the Morton search only the images its ghost rule keeps (code -1 for
    the rest, morton_ghost.cuh:28-50), as the oracle decides them;
  * past pi (w2_wide_3d) the rule matters: indexing every image would change many rows;
  * every neighbour row bit-identical to the oracle's restatement of the reference heap with its
    dedup (gdo_knn_brute_images, index_heap.cuh:112-176) over the device's own sites, and the kept
    K-th d^2 bit-identical; the radius-bounded search gives the same rows;
  * against the reference's CUDA build of the same model (oracle/_ref/collide_w*_65536: its
    col_site_init with images, its KD tree or Morton ghost index, and col_cache_get):
      - the same set of indexed images (every image for KD, the ghost records for Morton), every
        image coordinate bit-identical to the reference's KD node or Morton ghost record of the same
        code, and every physical site too;
      - the KD rows as sets (the reference writes heap order), the Morton rows in order, every
        measure to 1e-12 relative;
      - on the Morton wedge, the collision operator leaves every particle as the reference's does
        (grain size and count to 1e-12 relative).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEDGES = ["w0_wedge_3d", "w1_narrow_2d", "w2_wide_3d"]


def _run(gd, cfg, p, radius_scale=None):
    import torch

    sw = gd.SwarmCollision(cfg, len(p))
    dp = gd.particles_to_device(p)
    codes, measure, kth = sw.knn(dp)
    site4, q, active = (t.cpu().numpy() for t in sw.get_sites())
    bounded = None
    if radius_scale is not None:
        radius = torch.from_numpy(q * np.float32(radius_scale)).to(dp.device)
        bc = torch.empty_like(codes)
        bk = torch.empty_like(kth)
        sw.col_cache_get_bounded(dp, radius, bc, None, bk, None)
        bounded = (bc.cpu().numpy(), bk.cpu().numpy())
    torch.cuda.synchronize()
    out = codes.cpu().numpy(), measure.cpu().numpy(), kth.cpu().numpy(), site4, q, active, bounded
    sw.close()
    return out


@pytest.mark.parametrize("workload", WEDGES)
def test_wedge_sites_and_rows_match_the_oracle(gd, cuda, workload):
    from gamedev_b200 import GD_SEARCH_MORTON, workloads
    from oracle import oracle

    n = 16384
    cfg = workloads.config(workload)
    p = workloads.particles(workload, n=n)
    codes, _, kth, site4, q, active, bounded = _run(gd, cfg, p, radius_scale=0.35)
    wedge, width, idm = gd.wedge_info(cfg)
    assert wedge and site4.shape == (3 * n, 4)
    code = site4[:, 3].view(np.int32)
    i = np.arange(n)
    assert np.array_equal(code[:n], 3 * i)
    present = np.ones((n, 2), bool)
    if cfg.search == GD_SEARCH_MORTON:
        # the Morton ghost rule keeps an image only near the seam it stands for; the decisions the
        # oracle makes farther than float rounding from q_max must agree
        present = np.stack([code[n:2 * n] != -1, code[2 * n:] != -1], axis=1)
        keep, margin = oracle.morton_ghosts(site4[:n], p[:, 0].astype(np.float32), float(q.max()),
                                            cfg.x_min, cfg.x_max)
        sure = np.abs(margin) > 1e-5
        assert sure.mean() > 0.999
        assert np.array_equal(present[sure], keep[sure]), int((present[sure] != keep[sure]).sum())
    for img in (1, 2):
        pr = present[:, img - 1]
        assert np.array_equal(code[img * n:(img + 1) * n][pr], (3 * i + img)[pr])
    for img, ang in ((1, -width), (2, width)):
        c, s = math.cos(ang), math.sin(ang)
        x, y = site4[:n, 0].astype(np.float64), site4[:n, 1].astype(np.float64)
        blk = site4[img * n:(img + 1) * n].astype(np.float64)
        r = np.hypot(x, y)
        assert np.abs(blk[:, 0] - (c * x - s * y)).max() <= 1e-6 * r.max()
        assert np.abs(blk[:, 1] - (s * x + c * y)).max() <= 1e-6 * r.max()
        assert np.array_equal(blk[:, 2], site4[:n, 2])
    q_dedup = float(q.max()) if cfg.search == GD_SEARCH_MORTON else -1.0
    want, wd2 = oracle.knn_brute_images(site4, n, q, active, cfg.n_k, idm, q_dedup)
    bad = np.nonzero((want != codes).any(axis=1))[0]
    assert bad.size == 0, (workload, int(bad.size), int(bad[0]), want[bad[0]][:8], codes[bad[0]][:8])
    act = active.astype(bool)
    if width > math.pi:
        # wider than pi, images far from both seams land among the physical sites: the rule drops
        # them (about a third of all images here, where q_max is large against the inner radii),
        # and with every image indexed many rows would change (about 30% of the active owners)
        assert (~present).mean() > 0.25
        every = site4.copy()
        every[n:2 * n, 3] = (3 * i + 1).astype(np.int32).view(np.float32)
        every[2 * n:, 3] = (3 * i + 2).astype(np.int32).view(np.float32)
        naive, _ = oracle.knn_brute_images(every, n, q, active, cfg.n_k, idm, q_dedup)
        assert (naive != want).any(axis=1)[act].mean() > 0.05
    kth_want = np.where(want >= 0, wd2, 0.0).max(axis=1).astype(np.float32)
    assert np.array_equal(kth_want[act].view(np.uint32), kth[act].view(np.uint32))
    # the rows reach images, and some owners have the dedup on (their K nearest here never hold two
    # images of one particle: test_dedup_replaces_a_held_image covers that)
    assert (codes[act] % 3 != 0).any()
    assert np.any(2.0 * (q_dedup if q_dedup >= 0 else q[act]) >= idm)
    # the radius-bounded search (walk first out to 0.35 q) gives the same rows
    assert np.array_equal(bounded[0], codes)
    assert np.array_equal(bounded[1].view(np.uint32), kth.view(np.uint32))


@pytest.mark.parametrize("search", ["kd", "morton"])
def test_dedup_replaces_a_held_image(gd, cuda, search):
    """A 0.002 rad sliver of 4096 particles: an owner's 32 nearest span several wedge widths, so
    two or three images of one particle fall inside its ball and the dedup must keep the nearer."""
    from gamedev_b200 import GD_SEARCH_KDTREE, GD_SEARCH_MORTON, workloads
    from oracle import oracle

    n, width = 4096, 0.002
    cfg = workloads.config("w1_narrow_2d")
    cfg.search = GD_SEARCH_KDTREE if search == "kd" else GD_SEARCH_MORTON
    cfg.x_min, cfg.x_max = 0.0, width
    p = workloads.particles("w1_narrow_2d", n=n)
    p[:, 0] *= width / 0.05  # azimuths into [0, width)
    codes, _, kth, site4, q, active, bounded = _run(gd, cfg, p, radius_scale=0.5)
    wedge, _, idm = gd.wedge_info(cfg)
    assert wedge
    q_dedup = float(q.max()) if search == "morton" else -1.0
    want, wd2 = oracle.knn_brute_images(site4, n, q, active, cfg.n_k, idm, q_dedup)
    bad = np.nonzero((want != codes).any(axis=1))[0]
    assert bad.size == 0, (search, int(bad.size), int(bad[0]), want[bad[0]][:8], codes[bad[0]][:8])
    act = active.astype(bool)
    kth_want = np.where(want >= 0, wd2, 0.0).max(axis=1).astype(np.float32)
    assert np.array_equal(kth_want[act].view(np.uint32), kth[act].view(np.uint32))
    # no row holds two images of one particle, and without the dedup many rows would
    kept = np.where(codes >= 0, codes // 3, -1 - np.arange(cfg.n_k)[None, :])
    assert all(len(set(r.tolist())) == cfg.n_k for r in kept[act])
    plain, _ = oracle.knn_brute_images(site4, n, q, active, cfg.n_k, -1.0)
    assert (plain != want).any(axis=1).sum() > n // 10
    assert np.array_equal(bounded[0], codes)
    assert np.array_equal(bounded[1].view(np.uint32), kth.view(np.uint32))


def _refc(workload, n):
    from oracle.ref import refcollide

    if not refcollide.available(workload, n):
        pytest.skip("oracle/_ref reference collision build absent (reference tree not mounted at build time)")
    return refcollide


def _mass(p):
    return float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())


@pytest.mark.parametrize("workload", WEDGES)
def test_wedge_images_and_rows_match_the_reference_build(gd, cuda, workload):
    from gamedev_b200 import GD_SEARCH_MORTON, workloads

    n = 65536
    refcollide = _refc(workload, n)
    cfg = workloads.config(workload)
    p = workloads.particles(workload, n=n)
    codes, measure, _, site4, _, active, _ = _run(gd, cfg, p)
    _, info = refcollide.run(workload, p, 1, 1.0, _mass(p), 0, timeout=600, neighbours=True, records=True)
    # every reference record (KD nodes; Morton points and ghosts) against our site of the same code
    rec = info["records"]
    rcode = rec[:, 3].view(np.int32)
    scode = site4[:, 3].view(np.int32)
    kept = scode != -1
    # the KD tree holds every image; the Morton ghost index exactly the images its ghost rule keeps
    # (morton_ghost.cuh:28-88), which are the ones this build indexes
    assert np.array_equal(np.sort(rcode), np.sort(scode[kept])), (workload, rcode.size, int(kept.sum()))
    pos = np.full(3 * n, -1, np.int64)
    pos[scode[kept]] = np.nonzero(kept)[0]
    ours = site4[pos[rcode], :3]
    same_site = (ours.view(np.uint32) == rec[:, :3].view(np.uint32)).all(axis=1)
    assert same_site.all(), (workload, int((~same_site).sum()), rcode[~same_site][:4])
    _, width, _ = gd.wedge_info(cfg)
    # images are present in the reference's records (far fewer past pi: only those near a seam)
    assert (rcode % 3 != 0).sum() > (n // 100 if width > math.pi else n // 10)
    # the neighbour cache
    rc, rm = info["codes"], info["measure"]
    if cfg.search == GD_SEARCH_MORTON:
        same = (rc == codes).all(axis=1)
    else:
        same = (np.sort(rc, axis=1) == np.sort(codes, axis=1)).all(axis=1)
    bad = np.nonzero(~same)[0]
    assert bad.size == 0, (workload, int(bad.size), int(bad[0]), np.sort(rc[bad[0]])[:8],
                           np.sort(codes[bad[0]])[:8])
    assert (codes[active.astype(bool)] % 3 != 0).any()
    assert np.allclose(measure, rm, rtol=1e-12, atol=0)


@pytest.mark.parametrize("workload", ["w1_narrow_2d", "w2_wide_3d"])
def test_morton_wedge_operator_matches_the_reference_per_particle(gd, cuda, workload):
    import torch

    from gamedev_b200 import workloads

    n = 65536
    refcollide = _refc(workload, n)
    cfg = workloads.config(workload)
    p = workloads.particles(workload, n=n, seed=21)
    # an operator giving the fastest owner about 2000 expected events at bath start
    sw = gd.SwarmCollision(cfg, n)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(n, seed=1)
    sw.evolve_collisions(dp, rng, 1.0e-12 * workloads.orbital_time(), _mass(p))
    rates = sw.owner_state()[0][:, 0].cpu().numpy()
    sw.close()
    duration = 2000.0 / rates.max()
    for seed in (1, 2):
        sw = gd.SwarmCollision(cfg, n)
        dp = gd.particles_to_device(p)
        rng = gd.rngstate_init(n, seed=seed)
        sw.evolve_collisions(dp, rng, duration, _mass(p))
        torch.cuda.synchronize()
        ours = dp.cpu().numpy()
        events = sw.last_operator_stats()
        sw.close()
        ref, _ = refcollide.run(workload, p, seed, duration, _mass(p), 1, timeout=600)
        same = (np.isclose(ours[:, 6], ref[:, 6], rtol=1e-12, atol=0)
                & np.isclose(ours[:, 7], ref[:, 7], rtol=1e-12, atol=0))
        assert same.all(), (seed, int((~same).sum()), events)
        assert (ours[:, 6] != p[:, 6]).any()  # the operator changed grains
