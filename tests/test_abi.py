"""CPU checks of the drop-in boundary: the C-ABI library loads, exports every symbol the public
headers declare, mirrors the reference's const_defs.cuh defaults and rejects invalid models
before touching a device."""

import ctypes as C
import math
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(gd_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(gd):
    lib = gd.load()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header(gd):
    from gamedev_b200 import _lib

    assert set(declared_symbols()) <= set(_lib.SIGNATURES), set(declared_symbols()) - set(_lib.SIGNATURES)


def test_config_defaults_match_reference_const_defs(gd):
    # inc/swarm/const_defs.cuh:30-168 (the values the reference compiles by default)
    cfg = gd.default_config()
    assert (cfg.G, cfg.M_S, cfg.R_0, cfg.S_0) == (1.0, 1.0, 1.0, 1.0)
    assert (cfg.n_x, cfg.n_y, cfg.n_z) == (100, 100, 1)
    assert cfg.x_min == -math.pi and cfg.x_max == math.pi
    assert (cfg.y_min, cfg.y_max) == (0.5, 1.5)
    assert (cfg.sigma_0, cfg.aspr_0, cfg.idx_p, cfg.idx_q) == (1.0e-2, 0.05, -1.0, -0.4)
    assert (cfg.alpha, cfg.nu) == (1.0e-4, 1.0e-5)
    assert cfg.reynolds_0 == 1.0e8 and cfg.m_mol == 2.3 * 1.66054e-24 and cfg.x_sec == 2.0e-15
    assert (cfg.stokes_0, cfg.rho_0) == (1.0e-3, 1.0)
    assert (cfg.coag_kernel, cfg.n_k, cfg.h_search, cfg.v_frag) == (0, 200, 1.0, 1.0)
    assert cfg.col_event_cap == 32
    assert (cfg.col_bin_x, cfg.col_bin_y, cfg.col_bin_z, cfg.col_bin_s, cfg.col_bin_min) == (8, 4, 2, 8, 64)
    assert (cfg.col_bath_max, cfg.col_bath_eps, cfg.col_bath_alpha) == (0.05, 0.02, 1.0e-3)
    assert (cfg.morton_leaf_target, cfg.morton_max_level) == (128, 20)


def test_python_config_defaults_equal_the_library_defaults(gd):
    """config_defaults() builds gd_config_default's values without loading the library (the
    benchmark's reference arm uses it); every field must agree bit for bit."""
    from gamedev_b200 import _lib

    native, py = gd.default_config(), _lib.config_defaults()
    for name, _ in _lib.GdConfig._fields_:
        a, b = getattr(native, name), getattr(py, name)
        assert a == b and type(a) is type(b), (name, a, b)


def test_workloads_do_not_load_the_library():
    """The reference arm builds its configuration and particles through workloads: that must not
    map libgd_b200.so."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, %r); from gamedev_b200 import workloads, _lib; "
            "workloads.config('c3_learned_3d'); workloads.particles('c0_plain_small', n=64); "
            "assert _lib._lib is None; "
            "assert 'libgd_b200' not in open('/proc/self/maps').read()" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


def test_rng_state_is_curand_xorwow_size(gd):
    assert gd.rng_state_bytes() == 48


@pytest.mark.parametrize(
    "overrides,n",
    [
        ({}, 0),
        ({}, -5),
        ({"n_k": 0}, 100),
        ({"n_k": 257}, 100),
        ({"coag_kernel": 4}, 100),
        ({}, 800_000_000),  # 3*N overflows int32 neighbour codes
        ({"n_x": 64, "x_min": -0.1, "x_max": 0.1}, 357_913_942),  # a wedge: 3N sites above 2^30
    ],
)
def test_create_rejects_invalid_models_without_a_device(gd, overrides, n):
    from gamedev_b200 import _lib

    cfg = gd.default_config(**overrides)
    h = C.c_void_p()
    st = gd.load().gd_create(C.byref(cfg), n, C.byref(h))
    assert st == 1 and not h.value  # GD_ERR_INVALID_ARGUMENT, no handle


def test_wedges_are_rejected_by_the_one_site_per_particle_paths(gd):
    """A wedge (n_x > 1, azimuth shorter than 2 pi) has three sites per particle: the batch and the
    fixed-scratch search refuse it before any device work; gd_create accepts it."""
    lib = gd.load()
    cfg = gd.default_config(n_x=64, x_min=-0.1, x_max=0.1)
    b = C.c_void_p()
    n_p, n_k = (C.c_int * 1)(1024), (C.c_int * 1)(16)
    assert lib.gd_batch_create(C.byref(cfg), 1, n_p, n_k, C.byref(b)) == 1 and not b.value
    msg = C.create_string_buffer(256)
    fake = C.c_void_p(256)  # never dereferenced: the call returns before any device work
    st = lib.gd_knn_static(C.byref(cfg), fake, 1024, fake, fake, fake, None, None, msg, 256)
    assert st == 1 and b"wedge" in msg.value


def test_null_arguments_are_rejected(gd):
    lib = gd.load()
    assert lib.gd_create(None, 10, None) == 1
    assert lib.gd_geometry_build(None, None) == 1
    assert lib.gd_knn(None, None, None, None, None) == 1
    assert lib.gd_collision_operator(None, None, None, 1.0, 1.0) == 1
    assert lib.gd_rng_init(None, 4, 1, None) == 1
    lib.gd_destroy(None)


def test_particle_record_is_reference_layout(gd):
    from gamedev_b200 import PARTICLE_DTYPE

    assert PARTICLE_DTYPE.itemsize == 64  # const_defs.cuh:194-203 with MULTISIZE


def test_misaligned_device_pointers_are_rejected_before_any_launch(gd):
    """RNG states and particle records hold doubles: a pointer off their 8-byte alignment (e.g. a
    byte-offset slice of a state buffer) would fault the first kernel that loads through it, so
    the entry points return GD_ERR_INVALID_ARGUMENT before touching the device."""
    lib = gd.load()
    odd = C.c_void_p(0x10000 + 4)  # never dereferenced: the check comes first
    assert lib.gd_rng_init(odd, 1, 1, None) == 1
    assert lib.gd_rng_uniforms(odd, 1, 1, C.c_void_p(0x20000), None) == 1
    assert lib.gd_rng_uniforms(C.c_void_p(0x20000), 1, 1, odd, None) == 1
