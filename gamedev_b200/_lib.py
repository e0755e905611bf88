"""ctypes binding of libgd_b200.so (the C ABI in include/gd_b200.h).

The shared library is loaded from this package directory.  There is no fallback: if the library
is missing or cannot be loaded, every entry point raises, so no CPU path can stand in for the
CUDA kernels.
"""

from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgd_b200.so"

GD_OK = 0
STATUS_NAMES = {
    0: "GD_OK",
    1: "GD_ERR_INVALID_ARGUMENT",
    2: "GD_ERR_CUDA",
    3: "GD_ERR_NONFINITE",
    4: "GD_ERR_CHAIN",
    5: "GD_ERR_CAPACITY",
    6: "GD_ERR_CONTINUATION_LIMIT",
    7: "GD_ERR_TIME_RESOLUTION",
    8: "GD_ERR_CONTROLLER",
    9: "GD_ERR_NOT_READY",
    10: "GD_ERR_OUT_OF_MEMORY",
    11: "GD_ERR_TIMEOUT",
    12: "GD_ERR_IO",
}
GD_SEARCH_KDTREE, GD_SEARCH_MORTON = 0, 1
GD_KERNEL_CONSTANT, GD_KERNEL_LINEAR, GD_KERNEL_PRODUCT, GD_KERNEL_CUSTOM = 0, 1, 2, 3


class GdConfig(C.Structure):
    """gd_config: the const_defs.cuh constants of one model."""

    _fields_ = [
        ("G", C.c_double), ("M_S", C.c_double), ("R_0", C.c_double), ("S_0", C.c_double),
        ("n_x", C.c_int), ("n_y", C.c_int), ("n_z", C.c_int),
        ("x_min", C.c_double), ("x_max", C.c_double), ("y_min", C.c_double), ("y_max", C.c_double),
        ("z_min", C.c_double), ("z_max", C.c_double),
        ("sigma_0", C.c_double), ("aspr_0", C.c_double), ("idx_p", C.c_double), ("idx_q", C.c_double),
        ("const_nu", C.c_int), ("nu", C.c_double), ("alpha", C.c_double),
        ("code_unit", C.c_int), ("reynolds_0", C.c_double), ("m_mol", C.c_double), ("x_sec", C.c_double),
        ("half_disk", C.c_int), ("const_st", C.c_int),
        ("stokes_0", C.c_double), ("rho_0", C.c_double),
        ("coag_kernel", C.c_int), ("n_k", C.c_int), ("h_search", C.c_double), ("v_frag", C.c_double),
        ("col_event_cap", C.c_int),
        ("col_bin_x", C.c_int), ("col_bin_y", C.c_int), ("col_bin_z", C.c_int), ("col_bin_s", C.c_int),
        ("col_bin_min", C.c_int),
        ("col_bath_max", C.c_double), ("col_bath_eps", C.c_double), ("col_bath_alpha", C.c_double),
        ("init_smin", C.c_double), ("init_smax", C.c_double),
        ("search", C.c_int), ("morton_leaf_target", C.c_int), ("morton_max_level", C.c_int),
    ]

    def to_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GdRunInfo(C.Structure):
    """gd_run_info: the model-directory settings variables.txt records beyond gd_config."""

    _fields_ = [
        ("multisize", C.c_int), ("transport", C.c_int), ("diffusion", C.c_int), ("radiation", C.c_int),
        ("pr_effect", C.c_int), ("visc_flow", C.c_int), ("importgas", C.c_int), ("log_output", C.c_int),
        ("save_max", C.c_int), ("out_base", C.c_int), ("col_bath_tpb", C.c_int),
        ("metal_z", C.c_double), ("schmidt_x", C.c_double), ("schmidt_r", C.c_double), ("schmidt_z", C.c_double),
        ("beta_0", C.c_double), ("kappa_0", C.c_double), ("t_beta", C.c_double), ("c_light", C.c_double),
        ("dt_out", C.c_double), ("dt_max", C.c_double), ("cfl_dyn", C.c_double),
    ]


class GdTuning(C.Structure):
    _fields_ = [("warps_per_block", C.c_int), ("prescan", C.c_int), ("walk_breadth_first", C.c_int),
                ("sort_bits", C.c_int), ("range_query", C.c_int)]


class GdOperatorStats(C.Structure):
    _fields_ = [("waves", C.c_int), ("chain_launches", C.c_int), ("owner_updates", C.c_longlong),
                ("events", C.c_longlong), ("min_duration", C.c_double), ("max_duration", C.c_double)]


PARTICLE_BYTES = 64

# every symbol include/gd_b200.h declares, with (restype, argtypes)
_P = C.c_void_p
SIGNATURES = {
    "gd_rng_state_bytes": (C.c_size_t, []),
    "gd_config_default": (None, [C.POINTER(GdConfig)]),
    "gd_create": (C.c_int, [C.POINTER(GdConfig), C.c_int, C.POINTER(_P)]),
    "gd_destroy": (None, [_P]),
    "gd_set_stream": (C.c_int, [_P, _P]),
    "gd_last_error": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "gd_error_detail": (C.c_longlong, [_P]),
    "gd_rng_init": (C.c_int, [_P, C.c_int, C.c_ulonglong, _P]),
    "gd_geometry_build": (C.c_int, [_P, _P]),
    "gd_knn": (C.c_int, [_P, _P, _P, _P, _P]),
    "gd_set_deferred_checks": (C.c_int, [_P, C.c_int]),
    "gd_batch_create": (C.c_int, [C.POINTER(GdConfig), C.c_int, _P, _P, C.POINTER(_P)]),
    "gd_batch_destroy": (None, [_P]),
    "gd_batch_set_stream": (C.c_int, [_P, _P]),
    "gd_batch_knn": (C.c_int, [_P, _P, _P, _P, _P]),
    "gd_batch_check": (C.c_int, [_P]),
    "gd_batch_collide": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "gd_batch_operator_stats": (C.c_int, [_P, C.c_int, C.POINTER(GdOperatorStats)]),
    "gd_batch_invalidate": (C.c_int, [_P]),
    "gd_batch_reset_controller": (C.c_int, [_P]),
    "gd_batch_last_error": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "gd_batch_error_detail": (C.c_longlong, [_P]),
    "gd_batch_launch_count": (C.c_longlong, [_P]),
    "gd_batch_set_tuning": (C.c_int, [_P, C.POINTER(GdTuning)]),
    "gd_get_tuning": (C.c_int, [_P, C.POINTER(GdTuning)]),
    "gd_set_tuning": (C.c_int, [_P, C.POINTER(GdTuning)]),
    "gd_autotune": (C.c_int, [_P, _P, _P, C.c_int, C.POINTER(GdTuning), C.POINTER(C.c_double)]),
    "gd_check_geometry": (C.c_int, [_P]),
    "gd_get_sites": (C.c_int, [_P, _P, _P, _P]),
    "gd_site_count": (C.c_int, [_P]),
    "gd_wedge_info": (C.c_int, [C.POINTER(GdConfig), C.POINTER(C.c_int), C.POINTER(C.c_float),
                                C.POINTER(C.c_float)]),
    "gd_knn_bounded": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "gd_drift_keplerian": (C.c_int, [_P, _P, C.c_double]),
    "gd_pair_rates": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, _P]),
    "gd_radius_model_create": (C.c_int, [C.c_ulonglong, C.c_double, C.POINTER(_P)]),
    "gd_radius_model_destroy": (None, [_P]),
    "gd_radius_features": (C.c_int, [_P, _P, _P, C.c_double, _P]),
    "gd_radius_model_train": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_float,
                                        C.POINTER(C.c_float), _P]),
    "gd_radius_model_gradient": (C.c_int, [_P, _P, _P, C.c_int, _P, C.POINTER(C.c_float), _P]),
    "gd_radius_model_calibrate": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.POINTER(C.c_float), _P]),
    "gd_radius_model_predict": (C.c_int, [_P, _P, C.c_int, _P, _P]),
    "gd_radius_model_check": (C.c_int, [_P]),
    "gd_controller_summary": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "gd_operator_log": (C.c_size_t, [_P, C.c_char_p, C.c_size_t]),
    "gd_operator_phase_seconds": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "gd_bath_rates": (C.c_int, [_P, _P, C.c_double, _P]),
    "gd_bath_chain": (C.c_int, [_P, _P, _P, C.c_double, C.c_double, C.POINTER(C.c_ulonglong)]),
    "gd_set_diagnostics": (C.c_int, [_P, C.c_int]),
    "gd_event_totals": (C.c_int, [_P, _P, _P]),
    "gd_frame_name": (C.c_int, [C.c_int, C.c_int, C.c_char_p, C.c_size_t]),
    "gd_particles_to_file_layout": (C.c_int, [C.POINTER(GdConfig), _P, C.c_int]),
    "gd_particles_from_file_layout": (C.c_int, [C.POINTER(GdConfig), _P, C.c_int]),
    "gd_save_checkpoint": (C.c_int, [C.POINTER(GdConfig), C.c_char_p, C.c_int, C.c_int, _P, C.c_int, _P]),
    "gd_save_variables": (C.c_int, [C.POINTER(GdConfig), C.POINTER(GdRunInfo), C.c_int, C.c_double, C.c_char_p]),
    "gd_load_checkpoint": (C.c_int, [C.POINTER(GdConfig), C.c_char_p, C.c_int, C.c_int, _P, C.c_int, _P]),
    "gd_radius_model_get": (C.c_int, [_P, _P, _P]),
    "gd_radius_model_set": (C.c_int, [_P, _P, _P]),
    "gd_get_cache": (C.c_int, [_P, _P, _P]),
    "gd_set_cache": (C.c_int, [_P, _P, _P]),
    "gd_space_bin": (C.c_int, [_P, _P, _P]),
    "gd_invalidate_geometry": (C.c_int, [_P]),
    "gd_reset_controller": (C.c_int, [_P]),
    "gd_check_operator": (C.c_int, [_P]),
    "gd_collision_operator": (C.c_int, [_P, _P, _P, C.c_double, C.c_double]),
    "gd_evolve_collisions": (C.c_int, [_P, _P, _P, C.c_double, C.c_double]),
    "gd_last_operator_stats": (C.c_int, [_P, C.POINTER(GdOperatorStats)]),
    "gd_launch_count": (C.c_longlong, [_P]),
    "gd_rng_uniforms": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "gd_get_owner_state": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "gd_knn_static": (C.c_int, [C.POINTER(GdConfig), _P, C.c_int, _P, _P, _P, _P,
                                C.POINTER(C.c_longlong), C.c_char_p, C.c_size_t]),
    "gd_set_clock": (C.c_int, [_P, C.c_double, C.c_double, C.c_double]),
    "gd_get_clock": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_int)]),
    "gd_dynamics_step": (C.c_int, [_P, C.POINTER(GdRunInfo), _P, _P]),
    "gd_step": (C.c_int, [_P, C.POINTER(GdRunInfo), _P, _P, C.c_double, _P]),
    "gd_check_step": (C.c_int, [_P]),
    # include/gd_b200_controller.h (host only)
    "gd_ctl_binmap": (C.c_int, [C.c_int, C.c_int, C.c_int, _P, _P]),
    "gd_ctl_choose_bath": (C.c_int, [C.POINTER(GdConfig), _P, C.c_int, C.c_double, C.c_double, _P, _P]),
    "gd_ctl_finish_bath": (C.c_int, [C.POINTER(GdConfig), _P, C.c_int, _P, _P]),
    "gd_ctl_schedule_create": (_P, [C.c_double, _P, C.c_int, _P, _P]),
    "gd_ctl_schedule_destroy": (None, [_P]),
    "gd_ctl_schedule_time": (C.c_ulonglong, [_P]),
    "gd_ctl_schedule_end": (C.c_ulonglong, [_P]),
    "gd_ctl_schedule_due": (C.c_int, [_P, C.c_ulonglong, _P]),
    "gd_ctl_schedule_adapt": (C.c_int, [_P, C.c_ulonglong, _P, C.c_int, _P, _P]),
    "gd_ctl_schedule_advance": (None, [_P, _P, C.c_int]),
    "gd_ctl_schedule_levels": (None, [_P, _P]),
}

_lib = None


def load() -> C.CDLL:
    """Load libgd_b200.so; raise if it is absent (build it with gamedev_b200.build.build())."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build the CUDA extension first "
                               "(python -c 'import gamedev_b200.build as b; b.build()')")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class GdError(RuntimeError):
    def __init__(self, status: int, message: str, detail: int):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message} (detail {detail})")
        self.status = status
        self.message = message
        self.detail = detail


# gd_config_default's values (gamedev_b200/csrc/gd_api.cu), restated so that a configuration can be
# built without loading the library (the reference arm of the benchmark must not map it);
# tests/test_abi.py checks that the two agree field by field
CONFIG_DEFAULTS = {
    "G": 1.0, "M_S": 1.0, "R_0": 1.0, "S_0": 1.0, "n_x": 100, "n_y": 100, "n_z": 1,
    "x_min": -math.pi, "x_max": math.pi, "y_min": 0.5, "y_max": 1.5, "z_min": 0.5 * math.pi,
    "z_max": 0.5 * math.pi, "sigma_0": 1.0e-2, "aspr_0": 0.05, "idx_p": -1.0, "idx_q": -0.4,
    "const_nu": 0, "nu": 1.0e-5, "alpha": 1.0e-4, "code_unit": 0, "reynolds_0": 1.0e8,
    "m_mol": 2.3 * 1.66054e-24, "x_sec": 2.0e-15, "half_disk": 0, "const_st": 0, "stokes_0": 1.0e-3,
    "rho_0": 1.0, "coag_kernel": GD_KERNEL_CONSTANT, "n_k": 200, "h_search": 1.0, "v_frag": 1.0,
    "col_event_cap": 32, "col_bin_x": 8, "col_bin_y": 4, "col_bin_z": 2, "col_bin_s": 8, "col_bin_min": 64,
    "col_bath_max": 0.05, "col_bath_eps": 0.02, "col_bath_alpha": 1.0e-3, "init_smin": 1.0, "init_smax": 1.0,
    "search": GD_SEARCH_KDTREE, "morton_leaf_target": 128, "morton_max_level": 20,
}


def config_defaults(**overrides) -> GdConfig:
    """gd_config_default's configuration built in Python, without loading libgd_b200.so."""
    cfg = GdConfig()
    for k, v in {**CONFIG_DEFAULTS, **overrides}.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


def default_config(**overrides) -> GdConfig:
    cfg = GdConfig()
    load().gd_config_default(C.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg
