"""Checkpoint formats against the reference's own writer and reader (CPU).

oracle/_ref/io_<model>_<n>/ref_io is the reference's host I/O (inc/swarm/swarm_host.cuh:
save_sam_as_velocity, load_velocity_as_sam, save_host_binary, load_host_binary, frame_num)
compiled from the GameDev tree against the model header mod/make_models.py writes for the same
configuration (oracle/ref/Makefile).  Bars:
  * frame names equal frame_num for indices below, at and above the 5-digit width and save_max;
  * the particle file the library's layout conversion produces is byte-identical to the file the
    reference writes for the same particles (random velocities, plus owners at R = 0 and y = 0);
  * reading a reference file back gives the reference's internal records bit for bit;
  * variables.txt from gd_save_variables is byte-identical to the one save_variable writes for the
    same model (the model header's constants come from workloads.config and workloads.run_info),
    also for v0_radial_units, the radial model with the other branches of the file: code units, a
    constant viscosity, radiation with the PR effect, viscous flow, logarithmic output; and for
    v1_polar_gas, radial-polar with an imported gas density.
The c0 shapes are 3D (polar velocities converted; KD search, transport and diffusion flags), the c1
shapes 2D (polar pinned to pi/2; Morton search).
"""

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
N = 65536
MODELS = ["c0_plain_small", "c1_multisize_2d"]


def _ref_io(model, n=N):
    exe = ROOT / "oracle" / "_ref" / f"io_{model}_{n}" / "ref_io"
    if not exe.exists():
        pytest.skip("oracle/_ref reference I/O build absent (reference tree not mounted at build time)")
    return exe


def _save_max(model):
    defs = (ROOT / "oracle" / "_ref" / f"io_{model}_{N}" / "model" / "const_defs.cuh").read_text()
    return int(re.search(r"SAVE_MAX\s*=\s*(\d+)", defs).group(1))


def _n(model):
    """Particles of the model's reference I/O build: N for the benchmark shapes, else the config's."""
    from gamedev_b200 import workloads

    return N if model in MODELS else workloads.CONFIGS[model]["n"]


def _particles(model, seed=7):
    from gamedev_b200 import workloads

    n = _n(model)
    p = workloads.particles(model, n=n, seed=seed).copy()
    rng = np.random.default_rng(seed)
    p[:, 3:6] = rng.normal(size=(n, 3)) * 1e-3  # angular velocities of both signs
    p[5, 1] = 0.0          # y = 0: R = 0 and no polar speed
    p[9, 2] = 0.0          # on the pole: R = y sin z = 0 in 3D
    return p


def _write_records(path, p):
    with open(path, "wb") as f:
        f.write(np.int32(len(p)).tobytes())
        f.write(np.ascontiguousarray(p, np.float64).tobytes())


@pytest.mark.parametrize("model", MODELS)
def test_frame_names_match_reference(gd, model):
    exe = _ref_io(model)
    save_max = _save_max(model)
    for idx in (0, 7, 12, 99999, 123456):
        want = subprocess.run([str(exe), "frame", str(idx)], capture_output=True, text=True, check=True).stdout.strip()
        assert gd.frame_name(idx, save_max) == want, idx
    assert gd.frame_name(3, 1234567) == "0000003"  # width follows the digits of save_max


@pytest.mark.parametrize("model", MODELS + ["v0_radial_units", "v1_polar_gas"])
def test_particle_file_bytes_match_reference(gd, model, tmp_path):
    """Also on the radial (N_X = N_Z = 1) and radial-polar (N_X = 1) models, where the azimuth is
    pinned to the domain centre on both sides of the conversion."""
    from gamedev_b200 import workloads

    exe = _ref_io(model, _n(model))
    cfg = workloads.config(model)
    p = _particles(model)
    _write_records(tmp_path / "in.bin", p)
    subprocess.run([str(exe), "save", str(tmp_path / "in.bin"), str(tmp_path / "ref.dat")], check=True)
    ours = gd.particles_to_file_layout(cfg, p)
    assert (tmp_path / "ref.dat").read_bytes() == ours.tobytes()
    # reading the reference's file back: the reference's internal records, bit for bit
    subprocess.run([str(exe), "load", str(tmp_path / "ref.dat"), str(tmp_path / "back.bin")], check=True)
    back_ref = np.frombuffer((tmp_path / "back.bin").read_bytes()[4:], np.float64).reshape(-1, 8)
    back = gd.particles_from_file_layout(cfg, np.frombuffer((tmp_path / "ref.dat").read_bytes(), np.float64))
    assert np.array_equal(back.view(np.uint64), back_ref.view(np.uint64))


def test_reference_reader_rejects_wrong_size(gd, tmp_path):
    exe = _ref_io(MODELS[0])
    (tmp_path / "short.dat").write_bytes(b"\0" * (64 * N - 64))
    r = subprocess.run([str(exe), "load", str(tmp_path / "short.dat"), str(tmp_path / "x.bin")])
    assert r.returncode != 0  # the size check the library's reader restates (GD_ERR_IO)


@pytest.mark.parametrize("model", MODELS + ["v0_radial_units", "v1_polar_gas"])
def test_variables_file_matches_reference(gd, model, tmp_path):
    from gamedev_b200 import workloads

    n = _n(model)
    exe = _ref_io(model, n)
    mass = 1.0e-4 * workloads.MSUN * 0.731  # any positive total dust mass
    ref, ours = tmp_path / "ref_variables.txt", tmp_path / "variables.txt"
    subprocess.run([str(exe), "variables", str(ref), repr(mass)], check=True)
    gd.save_variables(workloads.config(model), workloads.run_info(model), n, mass, str(ours))
    want = ref.read_bytes()
    assert b"[SWARM_DTYPE]" in want and b"LAMBDA_0" in want
    assert ours.read_bytes() == want, "\n".join(
        f"{a!r} != {b!r}" for a, b in zip(ours.read_text().splitlines(), ref.read_text().splitlines()) if a != b)

