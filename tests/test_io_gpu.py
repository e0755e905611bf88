"""Checkpoints written and read through device memory, and an exact resume from them.

Bars:
  * gd_save_checkpoint writes the particle file the reference writes (the host conversion pinned
    byte for byte by tests/test_io.py) and the raw RNG states; gd_load_checkpoint restores the
    device particles and RNG states bit for bit;
  * a truncated or missing file is GD_ERR_IO and leaves the device buffers untouched;
  * resuming is exact: operator, checkpoint, a fresh handle that loads it, operator equals
    operator, controller reset (the reference resets the controller at every output boundary,
    swarm_runtime.cu:490-496), operator on one handle, for every particle and RNG state.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(gd, model="c1_multisize_2d", n=1 << 15, seed=3):
    from gamedev_b200 import workloads

    cfg = workloads.config(model)
    p = workloads.particles(model, n=n, seed=seed)
    p[:, 3:6] = np.random.default_rng(seed).normal(size=(n, 3)) * 1e-3
    mass = float((p[:, 7] * math.pi * p[:, 6] ** 3 / 6.0).sum())
    return cfg, p, mass


def test_checkpoint_round_trip(gd, cuda, tmp_path):
    import torch

    cfg, p, _ = _setup(gd)
    n = len(p)
    dp = gd.particles_to_device(p)
    rng = gd.rngstate_init(n, seed=9)
    prefix = str(tmp_path) + "/"
    gd.save_checkpoint(cfg, prefix, 4, dp, rng, save_max=10)
    name = gd.frame_name(4, 10)
    raw = (tmp_path / f"particle_{name}.dat").read_bytes()
    assert raw == gd.particles_to_file_layout(cfg, p).tobytes()
    assert (tmp_path / f"rngstate_{name}.dat").read_bytes() == rng.cpu().numpy().tobytes()
    dq = torch.zeros_like(dp)
    rq = torch.zeros_like(rng)
    gd.load_checkpoint(cfg, prefix, 4, dq, rq, save_max=10)
    torch.cuda.synchronize()
    back = gd.particles_from_file_layout(cfg, gd.particles_to_file_layout(cfg, p))
    assert np.array_equal(dq.cpu().numpy().view(np.uint64), back.view(np.uint64))
    assert torch.equal(rq, rng)


def test_checkpoint_size_mismatch_is_an_io_error(gd, cuda, tmp_path):
    import torch

    cfg, p, _ = _setup(gd)
    n = len(p)
    dp = gd.particles_to_device(p)
    prefix = str(tmp_path) + "/"
    gd.save_checkpoint(cfg, prefix, 1, dp, None, save_max=10)
    f = tmp_path / f"particle_{gd.frame_name(1, 10)}.dat"
    f.write_bytes(f.read_bytes()[:-64])  # one record short
    dq = torch.full_like(dp, 5.0)
    with pytest.raises(gd.GdError) as e:
        gd.load_checkpoint(cfg, prefix, 1, dq, None, save_max=10)
    assert e.value.status == 12
    assert torch.equal(dq, torch.full_like(dp, 5.0))
    with pytest.raises(gd.GdError) as e:
        gd.load_checkpoint(cfg, prefix, 2, dq, None, save_max=10)  # no such frame
    assert e.value.status == 12


@pytest.mark.parametrize("model", ["c1_multisize_2d", "c0_plain_small"])
def test_resume_from_checkpoint_is_exact(gd, cuda, tmp_path, model):
    import torch

    from gamedev_b200 import workloads

    cfg, p, mass = _setup(gd, model)
    n = len(p)
    # operator length: about 20 expected events for the fastest owner at the bath-start rates
    sw0 = gd.SwarmCollision(cfg, n)
    sw0.evolve_collisions(gd.particles_to_device(p), gd.rngstate_init(n, seed=1), 1.0e-12 * workloads.orbital_time(),
                          mass)
    dur = 20.0 / float(sw0.owner_state()[0][:, 0].max().item())
    sw0.close()
    # uninterrupted: two operators on one handle, the controller reset between them
    sw = gd.SwarmCollision(cfg, n)
    da = gd.particles_to_device(p)
    ra = gd.rngstate_init(n, seed=5)
    sw.evolve_collisions(da, ra, dur, mass)
    prefix = str(tmp_path) + "/"
    gd.save_checkpoint(cfg, prefix, 1, da, ra, save_max=10)
    sw.reset_controller()
    sw.evolve_collisions(da, ra, dur, mass)
    torch.cuda.synchronize()
    events = sw.last_operator_stats()["events"]
    sw.close()
    # resumed: a fresh handle reads the checkpoint and runs the second operator
    sw2 = gd.SwarmCollision(cfg, n)
    db = torch.zeros_like(da)
    rb = torch.zeros_like(ra)
    gd.load_checkpoint(cfg, prefix, 1, db, rb, save_max=10)
    sw2.evolve_collisions(db, rb, dur, mass)
    torch.cuda.synchronize()
    assert events > 0
    assert sw2.last_operator_stats()["events"] == events
    # the file layout pins inactive coordinates and round-trips velocities through R; the collision
    # path reads positions, sizes and numbers only, which the files carry unchanged
    assert torch.equal(da[:, 6:8], db[:, 6:8])
    # RNG states compared as streams (member-wise state copies need not keep struct padding)
    assert torch.equal(gd.rng_uniforms(ra, n, 4), gd.rng_uniforms(rb, n, 4))
    sw2.close()
