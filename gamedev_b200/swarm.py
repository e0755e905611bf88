"""Host-side mirror of the reference's swarm collision interface over the C ABI.

The names follow the reference's operator surface (src/swarm/swarm_runtime.cu:331-471,
inc/swarm/_col_chain.cuh:108): ``col_site_init`` + index build, ``col_cache_get``,
``evolve_local_collisions``, ``evolve_collisions``, ``invalidate_col_geometry`` and
``rngstate_init``.  Device memory comes from torch (plumbing only); every computation runs in
libgd_b200.so.  Errors raise :class:`GdError` carrying the reference's error meaning.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import GdConfig, GdError, GdOperatorStats

# gd_particle / reference `struct swarm` with MULTISIZE: 8 doubles
PARTICLE_FIELDS = ["x", "y", "z", "lx", "vy", "lz", "par_size", "par_numr"]
PARTICLE_DTYPE = np.dtype([(f, "<f8") for f in PARTICLE_FIELDS])


def _torch():
    import torch

    return torch


def _ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class SwarmCollision:
    """One swarm of n_p representative particles bound to a libgd_b200 handle."""

    def __init__(self, cfg: GdConfig, n_p: int):
        self.lib = _lib.load()
        self.cfg = cfg
        self.n_p = int(n_p)
        self.n_k = int(cfg.n_k)
        h = C.c_void_p()
        st = self.lib.gd_create(C.byref(cfg), self.n_p, C.byref(h))
        if st != _lib.GD_OK:
            raise GdError(st, "gd_create failed", 0)
        self.h = h
        self.lib.gd_set_stream(self.h, _stream())

    def close(self):
        if getattr(self, "h", None):
            self.lib.gd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != _lib.GD_OK:
            buf = C.create_string_buffer(512)
            self.lib.gd_last_error(self.h, buf, 512)
            raise GdError(st, buf.value.decode(), int(self.lib.gd_error_detail(self.h)))

    # ---- geometry stage -------------------------------------------------------------------
    def col_site_init(self, particles):
        """col_site_init + index build (swarm_runtime.cu:376-409)."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_geometry_build(self.h, C.c_void_p(_ptr(particles))))

    def tuning(self) -> dict:
        t = _lib.GdTuning()
        self._check(self.lib.gd_get_tuning(self.h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in t._fields_}

    def set_tuning(self, **kw):
        t = _lib.GdTuning(**{**self.tuning(), **kw})
        self._check(self.lib.gd_set_tuning(self.h, C.byref(t)))

    def autotune(self, particles, radius=None, tune_sort: bool = True):
        """gd_autotune on these particles (and proposed radii): returns (tuning dict, query ms)."""
        self.lib.gd_set_stream(self.h, _stream())
        t = _lib.GdTuning()
        ms = C.c_double(0.0)
        self._check(self.lib.gd_autotune(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(radius)),
                                         1 if tune_sort else 0, C.byref(t), C.byref(ms)))
        return {f: getattr(t, f) for f, _ in t._fields_}, float(ms.value)

    def set_deferred_checks(self, on: bool = True):
        """Defer the non-finite screen of col_site_init to check_geometry(), so a build + query
        sequence makes no host synchronisation (needed to capture it in a CUDA graph)."""
        self._check(self.lib.gd_set_deferred_checks(self.h, 1 if on else 0))

    def check_geometry(self):
        """Read the deferred non-finite screen of the last build; raises GdError on a bad particle."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_check_geometry(self.h))

    def col_cache_get(self, particles, codes=None, measure=None, kth_d2=None):
        """col_cache_get (_col_cache.cuh:15-159): fills codes [n_p, n_k] int32, measure [n_p] f64."""
        self._check(self.lib.gd_knn(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(codes)),
                                    C.c_void_p(_ptr(measure)), C.c_void_p(_ptr(kth_d2))))

    def col_cache_get_bounded(self, particles, radius=None, codes=None, measure=None, kth_d2=None, stats=None):
        """Radius-bounded exact top-K (gd_knn_bounded); radius [n_p] float32 by particle index or
        None; stats a uint64 [4] device tensor (leaves, nodes, offers, fallbacks) or None."""
        self._check(self.lib.gd_knn_bounded(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(radius)),
                                            C.c_void_p(_ptr(codes)), C.c_void_p(_ptr(measure)),
                                            C.c_void_p(_ptr(kth_d2)), C.c_void_p(_ptr(stats))))

    def knn(self, particles):
        """Geometry + exact top-K into fresh torch tensors: (codes, measure, kth_d2)."""
        torch = _torch()
        dev = particles.device
        codes = torch.empty((self.n_p, self.n_k), dtype=torch.int32, device=dev)
        measure = torch.empty(self.n_p, dtype=torch.float64, device=dev)
        kth = torch.empty(self.n_p, dtype=torch.float32, device=dev)
        self.col_site_init(particles)
        self.col_cache_get(particles, codes, measure, kth)
        return codes, measure, kth

    def build_cache(self, particles):
        """Geometry + top-K into the handle's own cache (used by the collision operator)."""
        self.col_site_init(particles)
        self.col_cache_get(particles)

    def get_sites(self):
        """Site-init outputs of the last geometry build: (site4 float32 [sites,4], q [n], active [n]);
        sites = n, or 3n for an azimuthal wedge (images n..2n-1 at -width, 2n..3n-1 at +width)."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        site4 = torch.empty((self.lib.gd_site_count(self.h), 4), dtype=torch.float32, device=dev)
        q = torch.empty(self.n_p, dtype=torch.float32, device=dev)
        active = torch.empty(self.n_p, dtype=torch.uint8, device=dev)
        self._check(self.lib.gd_get_sites(self.h, C.c_void_p(site4.data_ptr()), C.c_void_p(q.data_ptr()),
                                          C.c_void_p(active.data_ptr())))
        return site4, q, active

    def get_cache(self, codes, measure):
        self._check(self.lib.gd_get_cache(self.h, C.c_void_p(_ptr(codes)), C.c_void_p(_ptr(measure))))

    def set_cache(self, codes, measure):
        self._check(self.lib.gd_set_cache(self.h, C.c_void_p(_ptr(codes)), C.c_void_p(_ptr(measure))))

    def col_space_bin(self, particles, spatial):
        self._check(self.lib.gd_space_bin(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(spatial))))

    def invalidate_col_geometry(self):
        self._check(self.lib.gd_invalidate_geometry(self.h))

    def reset_controller(self):
        self._check(self.lib.gd_reset_controller(self.h))

    def set_diagnostics(self, on: bool = True):
        """COL_DIAGNOSTICS event bookkeeping per operator (gd_set_diagnostics)."""
        self._check(self.lib.gd_set_diagnostics(self.h, 1 if on else 0))

    def event_totals(self):
        """(counts [7] uint64, log_mass [7] float64) of the last operator's events per outcome
        category (gd_event_totals)."""
        counts = np.zeros(7, np.uint64)
        log_mass = np.zeros(7, np.float64)
        self._check(self.lib.gd_event_totals(self.h, C.c_void_p(counts.ctypes.data), C.c_void_p(log_mass.ctypes.data)))
        return counts, log_mass

    def controller_summary(self) -> dict:
        """COL_DIAGNOSTICS controller summary of the current output interval (gd_controller_summary),
        parsed from the JSON the reference's save_col_controller writes."""
        import json

        n = self.lib.gd_controller_summary(self.h, None, 0)
        buf = C.create_string_buffer(n + 1)
        self.lib.gd_controller_summary(self.h, buf, n + 1)
        return json.loads(buf.value.decode())

    def operator_log(self) -> list:
        """COL_DIAGNOSTICS per-operator log (gd_operator_log): one parsed JSON line per operator run
        with diagnostics on, in the reference's collision_local_*.jsonl format."""
        import json

        n = self.lib.gd_operator_log(self.h, None, 0)
        buf = C.create_string_buffer(n + 1)
        self.lib.gd_operator_log(self.h, buf, n + 1)
        return [json.loads(line) for line in buf.value.decode().splitlines() if line.strip()]

    def operator_phase_seconds(self) -> dict:
        """gd_operator_phase_seconds: device seconds of the logged operators by phase."""
        out = (C.c_double * 4)()
        self._check(self.lib.gd_operator_phase_seconds(self.h, out))
        return {"rates": out[0], "events": out[1], "audit": out[2], "operators": out[3]}

    # ---- collision operator ---------------------------------------------------------------
    def evolve_local_collisions(self, particles, rng, duration: float, total_dust_mass: float):
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_collision_operator(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng)),
                                                   float(duration), float(total_dust_mass)))

    def check_operator(self):
        """gd_check_operator: the status, statistics and bath records of the operators a captured
        CUDA graph ran (raises GdError with the first error any of them met)."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_check_operator(self.h))

    def evolve_collisions(self, particles, rng, duration: float, total_dust_mass: float):
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_evolve_collisions(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng)),
                                                  float(duration), float(total_dust_mass)))

    def owner_state(self):
        """(cached [n,4], time [n], events [n], size_old [n], numr_old [n]) of the last operator."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        cached = torch.empty((self.n_p, 4), dtype=torch.float64, device=dev)
        time = torch.empty(self.n_p, dtype=torch.float64, device=dev)
        events = torch.empty(self.n_p, dtype=torch.int32, device=dev)
        size_old = torch.empty(self.n_p, dtype=torch.float64, device=dev)
        numr_old = torch.empty(self.n_p, dtype=torch.float64, device=dev)
        self._check(self.lib.gd_get_owner_state(self.h, *(C.c_void_p(t.data_ptr()) for t in
                                                          (cached, time, events, size_old, numr_old))))
        return cached, time, events, size_old, numr_old

    def bath_rates(self, particles, total_mass: float, out=None):
        """gd_bath_rates: every owner's bath-start rate moments [n, 4] on the current cache."""
        torch = _torch()
        if out is None:
            out = torch.empty((self.n_p, 4), dtype=torch.float64, device=particles.device)
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_bath_rates(self.h, C.c_void_p(_ptr(particles)), float(total_mass),
                                           C.c_void_p(_ptr(out))))
        return out

    def bath_chain(self, particles, rng, total_mass: float, bath: float) -> int:
        """gd_bath_chain: one frozen bath of `bath` seconds for every owner, eagerly; returns the
        number of events.  The particles and RNG streams advance in place."""
        events = C.c_ulonglong(0)
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_bath_chain(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng)),
                                           float(total_mass), float(bath), C.byref(events)))
        return int(events.value)

    def pair_rates(self, particles, owner_ids, total_mass: float):
        """Per-pair bath-start terms [count, n_k, 5] = rate, rate*mean, rate*second, maximum, speed."""
        torch = _torch()
        count = int(owner_ids.shape[0])
        out = torch.empty((count, self.n_k, 5), dtype=torch.float64, device=particles.device)
        self._check(self.lib.gd_pair_rates(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(owner_ids)), count,
                                           float(total_mass), C.c_void_p(_ptr(out))))
        return out

    def launch_count(self) -> int:
        return int(self.lib.gd_launch_count(self.h))

    def last_operator_stats(self) -> dict:
        s = GdOperatorStats()
        self._check(self.lib.gd_last_operator_stats(self.h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}


    # ---- learned radius -------------------------------------------------------------------
    def drift_keplerian(self, particles, dt: float):
        """Keplerian azimuthal advance (gd_drift_keplerian); invalidates the geometry."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_drift_keplerian(self.h, C.c_void_p(_ptr(particles)), float(dt)))

    # ---- the Strang step (gd_step) -------------------------------------------------------------
    def set_clock(self, clock_sim: float = 0.0, clock_out: float = 0.0, dt_out: float = 1.0):
        """gd_set_clock: the time loop's device clocks and the output interval."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_set_clock(self.h, float(clock_sim), float(clock_out), float(dt_out)))

    def clock(self) -> dict:
        """gd_get_clock: clock_sim, clock_out, the last step's dt and the steps taken."""
        a, b, c, k = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_get_clock(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(k)))
        return {"clock_sim": a.value, "clock_out": b.value, "dt": c.value, "steps": k.value}

    def dynamics_step(self, run, particles, rng):
        """gd_dynamics_step: the timestep and D(dt/2) T(dt) D(dt/2), without collisions."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_dynamics_step(self.h, C.byref(run), C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng))))

    def step(self, run, particles, rng, total_dust_mass: float, radius_model=None):
        """gd_step: one Strang step C(dt/2) D(dt/2) T(dt) D(dt/2) C(dt/2); radius_model (a
        RadiusModel) seeds every geometry rebuild after the first with the learned proposal."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_step(self.h, C.byref(run), C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng)),
                                     float(total_dust_mass), radius_model.h if radius_model else None))

    def check_step(self):
        """gd_check_step: after a replay of captured steps, the non-finite screen of the last
        geometry build, else the first error of their collision operators (raises GdError)."""
        self.lib.gd_set_stream(self.h, _stream())
        self._check(self.lib.gd_check_step(self.h))

    def radius_features(self, particles, prev_kth_d2, total_mass: float, out=None):
        """Learned-radius features [n_p, 8] of the current geometry (gd_radius_features)."""
        torch = _torch()
        if out is None:
            out = torch.zeros((self.n_p, 8), dtype=torch.float32, device=particles.device)
        self._check(self.lib.gd_radius_features(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(prev_kth_d2)),
                                                float(total_mass), C.c_void_p(_ptr(out))))
        return out


class RadiusModel:
    """The learned search-radius network (gd_radius_model_*); every computation is a libgd_b200
    kernel."""

    N_PARAMS = 4801

    def __init__(self, R_0: float, seed: int = 1):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.gd_radius_model_create(C.c_ulonglong(seed), float(R_0), C.byref(h))
        if st != _lib.GD_OK:
            raise GdError(st, "gd_radius_model_create failed", 0)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.gd_radius_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != _lib.GD_OK:
            raise GdError(st, what, 0)

    def train(self, features, kth_d2, iterations: int, batch: int = 16384, lr: float = 1e-3) -> float:
        loss = C.c_float(0.0)
        self._check(self.lib.gd_radius_model_train(self.h, C.c_void_p(features.data_ptr()),
                                                   C.c_void_p(kth_d2.data_ptr()), int(features.shape[0]),
                                                   int(iterations), int(batch), float(lr), C.byref(loss), _stream()),
                    "gd_radius_model_train")
        return float(loss.value)

    def gradient(self, features, kth_d2):
        torch = _torch()
        g = torch.empty(self.N_PARAMS, dtype=torch.float32, device=features.device)
        loss = C.c_float(0.0)
        self._check(self.lib.gd_radius_model_gradient(self.h, C.c_void_p(features.data_ptr()),
                                                      C.c_void_p(kth_d2.data_ptr()), int(features.shape[0]),
                                                      C.c_void_p(g.data_ptr()), C.byref(loss), _stream()),
                    "gd_radius_model_gradient")
        return g, float(loss.value)

    def calibrate(self, features, kth_d2, quantile: float = 0.999) -> float:
        m = C.c_float(0.0)
        self._check(self.lib.gd_radius_model_calibrate(self.h, C.c_void_p(features.data_ptr()),
                                                       C.c_void_p(kth_d2.data_ptr()), int(features.shape[0]),
                                                       float(quantile), C.byref(m), _stream()),
                    "gd_radius_model_calibrate")
        return float(m.value)

    def predict(self, features, out=None):
        torch = _torch()
        if out is None:
            out = torch.empty(features.shape[0], dtype=torch.float32, device=features.device)
        self._check(self.lib.gd_radius_model_predict(self.h, C.c_void_p(features.data_ptr()), int(features.shape[0]),
                                                     C.c_void_p(out.data_ptr()), _stream()),
                    "gd_radius_model_predict")
        return out

    def check(self):
        """Synchronise and raise if a tensor-core forward stopped at a timed-out wait."""
        self._check(self.lib.gd_radius_model_check(self.h), "gd_radius_model_check")

    def get(self):
        p = np.zeros(self.N_PARAMS, np.float32)
        norm = np.zeros(17, np.float32)
        self._check(self.lib.gd_radius_model_get(self.h, p.ctypes.data, norm.ctypes.data), "gd_radius_model_get")
        return p, norm

    def set(self, params=None, norm=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        self._check(self.lib.gd_radius_model_set(self.h, None if p is None else p.ctypes.data,
                                                 None if nm is None else nm.ctypes.data), "gd_radius_model_set")


def rng_state_bytes() -> int:
    return int(_lib.load().gd_rng_state_bytes())


def wedge_info(cfg):
    """(wedge, width, image_dist_min) the search uses for cfg (gd_wedge_info): X_WEDGE, the images'
    rotation angle and _get_image_dist_min (-1 without a wedge)."""
    w, width, idm = C.c_int(), C.c_float(), C.c_float()
    r = _lib.load().gd_wedge_info(C.byref(cfg), C.byref(w), C.byref(width), C.byref(idm))
    if r != _lib.GD_OK:
        raise GdError(r, "gd_wedge_info failed", 0)
    return bool(w.value), float(width.value), float(idm.value)


def rngstate_init(n: int, seed: int = 1, device="cuda:0"):
    """rngstate_init (src/swarm/rngstate_init.cu:11-18): curand_init(seed, i, 0) per particle."""
    torch = _torch()
    st = torch.empty(n * rng_state_bytes(), dtype=torch.uint8, device=device)
    r = _lib.load().gd_rng_init(C.c_void_p(st.data_ptr()), int(n), C.c_ulonglong(seed), _stream())
    if r != _lib.GD_OK:
        raise GdError(r, "gd_rng_init failed", 0)
    return st


def rng_uniforms(rng, n: int, count: int):
    """The next `count` chain deviates of every particle's stream, drawn from copies (rng unchanged)."""
    torch = _torch()
    out = torch.empty((n, count), dtype=torch.float64, device=rng.device)
    r = _lib.load().gd_rng_uniforms(C.c_void_p(rng.data_ptr()), int(n), int(count), C.c_void_p(out.data_ptr()),
                                    _stream())
    if r != _lib.GD_OK:
        raise GdError(r, "gd_rng_uniforms failed", 0)
    return out


def particles_to_device(arr: np.ndarray, device="cuda:0"):
    """Structured or (n, 8) float64 host array -> contiguous (n, 8) float64 device tensor."""
    torch = _torch()
    a = np.ascontiguousarray(arr).view(np.float64).reshape(-1, 8)
    return torch.from_numpy(a.copy()).to(device)


def _io_check(status: int, what: str):
    if status != 0:
        raise GdError(status, what, 0)


def frame_name(idx_file: int, save_max: int) -> str:
    """The frame number of the reference's file names: idx_file zero padded to max(5, digits of
    save_max)."""
    buf = C.create_string_buffer(32)
    _io_check(_lib.load().gd_frame_name(int(idx_file), int(save_max), buf, len(buf)), "gd_frame_name")
    return buf.value.decode()


def particles_to_file_layout(cfg: GdConfig, arr: np.ndarray) -> np.ndarray:
    """Host particle records (n, 8) float64 in the internal layout -> a new array in the layout of
    the reference's particle files (linear azimuthal and polar speeds)."""
    a = np.ascontiguousarray(arr, np.float64).reshape(-1, 8).copy()
    _io_check(_lib.load().gd_particles_to_file_layout(C.byref(cfg), C.c_void_p(a.ctypes.data), a.shape[0]),
              "gd_particles_to_file_layout")
    return a


def particles_from_file_layout(cfg: GdConfig, arr: np.ndarray) -> np.ndarray:
    """The inverse of particles_to_file_layout, as the reference converts after reading a file."""
    a = np.ascontiguousarray(arr, np.float64).reshape(-1, 8).copy()
    _io_check(_lib.load().gd_particles_from_file_layout(C.byref(cfg), C.c_void_p(a.ctypes.data), a.shape[0]),
              "gd_particles_from_file_layout")
    return a


def save_checkpoint(cfg: GdConfig, prefix: str, idx_file: int, particles, rng=None, save_max: int = 0):
    """Write <prefix>particle_<frame>.dat (and rngstate_<frame>.dat when rng is given) from device
    tensors, in the reference's formats."""
    _io_check(_lib.load().gd_save_checkpoint(C.byref(cfg), str(prefix).encode(), int(idx_file), int(save_max),
                                             C.c_void_p(particles.data_ptr()), int(particles.shape[0]),
                                             C.c_void_p(rng.data_ptr() if rng is not None else None)),
              "gd_save_checkpoint")


def load_checkpoint(cfg: GdConfig, prefix: str, idx_file: int, particles, rng=None, save_max: int = 0):
    """Read a frame written by the reference (or by save_checkpoint) into device tensors of the
    right sizes; raises GdError(GD_ERR_IO) on a missing file or a size mismatch."""
    _io_check(_lib.load().gd_load_checkpoint(C.byref(cfg), str(prefix).encode(), int(idx_file), int(save_max),
                                             C.c_void_p(particles.data_ptr()), int(particles.shape[0]),
                                             C.c_void_p(rng.data_ptr() if rng is not None else None)),
              "gd_load_checkpoint")


def save_variables(cfg: GdConfig, run, n_p: int, total_dust_mass: float, path: str):
    """Write the run's variables.txt as the reference's save_variable does (gd_save_variables);
    `run` is a GdRunInfo with the model directory's other settings."""
    _io_check(_lib.load().gd_save_variables(C.byref(cfg), C.byref(run), int(n_p), float(total_dust_mass),
                                            str(path).encode()), "gd_save_variables")


STATIC_MAX_PARTICLES = 1 << 16  # gd_knn_static's fixed scratch


def knn_static(cfg: GdConfig, particles, codes, measure, kth):
    """Exact top-K through gd_knn_static, which allocates no device memory: for callers that may
    not call cudaMalloc while they run (a host that owns the whole device through its own pool, or
    a time loop that cannot take the synchronisation an allocation can cause).  Its scratch is a
    fixed 4.4 MB device array, so at most 65536 particles.  The caller provides the outputs; calls
    whose GPU work overlaps on one device race on the shared scratch."""
    torch = _torch()
    n = int(particles.shape[0])
    want = ((codes, torch.int32, (n, int(cfg.n_k))), (measure, torch.float64, (n,)), (kth, torch.float32, (n,)))
    for t, dtype, shape in want:
        if (t.dtype != dtype or tuple(t.shape) != shape or not t.is_contiguous()
                or t.device != particles.device):
            raise ValueError(f"knn_static output must be a contiguous {dtype} tensor of shape {shape} on "
                             f"{particles.device}, got {t.dtype} {tuple(t.shape)} on {t.device}")
    if not particles.is_cuda or not particles.is_contiguous():
        raise ValueError("knn_static particles must be a contiguous device tensor")
    detail = C.c_longlong(0)
    msg = C.create_string_buffer(512)
    r = _lib.load().gd_knn_static(C.byref(cfg), C.c_void_p(particles.data_ptr()), n, C.c_void_p(codes.data_ptr()),
                                  C.c_void_p(measure.data_ptr()), C.c_void_p(kth.data_ptr()), _stream(),
                                  C.byref(detail), msg, len(msg))
    if r != _lib.GD_OK:
        raise GdError(r, msg.value.decode(errors="replace"), int(detail.value))


class SwarmBatch:
    """Many independent swarms (uneven n_p and n_k, shared model constants) searched per call:
    per-swarm geometry builds side by side and one persistent top-K launch (gd_batch_*).  Buffers
    are concatenated swarm by swarm; `rows(t, s)` slices swarm s out of a concatenated result."""

    def __init__(self, cfg: GdConfig, sizes, ks):
        self.lib = _lib.load()
        self.sizes = [int(v) for v in sizes]
        self.ks = [int(v) for v in ks]
        self.S = len(self.sizes)
        n = (C.c_int * self.S)(*self.sizes)
        k = (C.c_int * self.S)(*self.ks)
        h = C.c_void_p()
        st = self.lib.gd_batch_create(C.byref(cfg), self.S, n, k, C.byref(h))
        if st != _lib.GD_OK:
            raise GdError(st, "gd_batch_create failed", 0)
        self.h = h
        self.part_off = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.codes_off = np.concatenate([[0], np.cumsum(np.array(self.sizes) * np.array(self.ks))]).astype(np.int64)

    def close(self):
        if getattr(self, "h", None):
            self.lib.gd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != _lib.GD_OK:
            buf = C.create_string_buffer(512)
            self.lib.gd_batch_last_error(self.h, buf, 512)
            raise GdError(st, buf.value.decode(), int(self.lib.gd_batch_error_detail(self.h)))

    def outputs(self, device="cuda"):
        torch = _torch()
        codes = torch.empty(int(self.codes_off[-1]), dtype=torch.int32, device=device)
        measure = torch.empty(int(self.part_off[-1]), dtype=torch.float64, device=device)
        kth = torch.empty(int(self.part_off[-1]), dtype=torch.float32, device=device)
        return codes, measure, kth

    def knn(self, particles, codes, measure, kth):
        """Geometry + exact top-K of every swarm (no host synchronisation; see check())."""
        self.lib.gd_batch_set_stream(self.h, _stream())
        self._check(self.lib.gd_batch_knn(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(codes)),
                                          C.c_void_p(_ptr(measure)), C.c_void_p(_ptr(kth))))

    def check(self):
        """The deferred non-finite screens of the last knn(), then the results of captured
        collide() calls; raises GdError (detail = index in the concatenated particle array, or the
        swarm of an operator error)."""
        self.lib.gd_batch_set_stream(self.h, _stream())
        self._check(self.lib.gd_batch_check(self.h))

    def collide(self, particles, rng, codes, measure, durations, total_dust_masses):
        """gd_batch_collide: every swarm's collision operator on the rows of the last knn(), side
        by side; durations and total_dust_masses per swarm."""
        d = (C.c_double * self.S)(*[float(v) for v in durations])
        m = (C.c_double * self.S)(*[float(v) for v in total_dust_masses])
        self.lib.gd_batch_set_stream(self.h, _stream())
        self._check(self.lib.gd_batch_collide(self.h, C.c_void_p(_ptr(particles)), C.c_void_p(_ptr(rng)),
                                              C.c_void_p(_ptr(codes)), C.c_void_p(_ptr(measure)), d, m))

    def reset_controller(self):
        """gd_batch_reset_controller: every swarm's bath controller memory afresh."""
        self.lib.gd_batch_set_stream(self.h, _stream())
        self._check(self.lib.gd_batch_reset_controller(self.h))

    def operator_stats(self, s: int) -> dict:
        st = GdOperatorStats()
        self._check(self.lib.gd_batch_operator_stats(self.h, int(s), C.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def codes_of(self, codes, s: int):
        a, b = int(self.codes_off[s]), int(self.codes_off[s + 1])
        return codes[a:b].view(self.sizes[s], self.ks[s])

    def rows_of(self, t, s: int):
        return t[int(self.part_off[s]):int(self.part_off[s + 1])]

    def set_tuning(self, warps_per_block=0, prescan=2, walk_breadth_first=1, sort_bits=0):
        t = _lib.GdTuning(warps_per_block, prescan, walk_breadth_first, sort_bits, 1)
        self._check(self.lib.gd_batch_set_tuning(self.h, C.byref(t)))

    def launch_count(self) -> int:
        return int(self.lib.gd_batch_launch_count(self.h))
