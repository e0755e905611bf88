"""ctypes binding of the reference's host-compiled collision code (oracle/_ref/libgd_ref_<model>.so,
built by oracle/ref/Makefile from the GameDev headers).  TEST INFRASTRUCTURE ONLY: a golden source
for the oracle and the library's host controller; absent where the reference tree is not mounted."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parents[1] / "_ref"
MODELS = ("phys", "code", "frag")


def available(model: str = "phys") -> bool:
    return (REF_DIR / f"libgd_ref_{model}.so").exists()


class RefHost:
    def __init__(self, model: str):
        lib = C.CDLL(str(REF_DIR / f"libgd_ref_{model}.so"))
        P, D, I = C.c_void_p, C.c_double, C.c_int
        sig = {
            "ref_n_k": (I, []),
            "ref_env": (None, [D, D, P]),
            "ref_pair_rate": (D, [D] * 9 + [P]),
            "ref_outcome_moments": (D, [D, D, I, P]),
            "ref_sample_outcome": (D, [D, D, I, D]),
            "ref_ball_measure": (D, [D, D, D]),
            "ref_raw_count": (I, []),
            "ref_binmap": (I, [P, I, P]),
            "ref_choose_bath": (I, [P, I, D, D, P, P]),
            "ref_finish_bath": (I, [P, I, P, P]),
            "ref_schedule_create": (P, [D, P, I, P, P]),
            "ref_schedule_destroy": (None, [P]),
            "ref_schedule_time": (C.c_ulonglong, [P]),
            "ref_schedule_end": (C.c_ulonglong, [P]),
            "ref_schedule_due": (I, [P, C.c_ulonglong, P]),
            "ref_schedule_adapt": (I, [P, C.c_ulonglong, P, I, P, P]),
            "ref_schedule_advance": (None, [P, P, I]),
            "ref_schedule_levels": (None, [P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        self.lib = lib
        self.model = model

    def env(self, y, z):
        out = np.zeros(8)
        self.lib.ref_env(y, z, out.ctypes.data)
        return out

    def pair_rate(self, yi, zi, yj, zj, si, sj, numr_j, lambda0, measure):
        v = C.c_double(0.0)
        r = self.lib.ref_pair_rate(yi, zi, yj, zj, si, sj, numr_j, lambda0, measure, C.byref(v))
        return r, v.value

    def outcome_moments(self, si, sj, high):
        out = np.zeros(3)
        f = self.lib.ref_outcome_moments(si, sj, int(high), out.ctypes.data)
        return f, out[0], out[1], out[2]

    def sample_outcome(self, si, sj, high, u):
        return self.lib.ref_sample_outcome(si, sj, int(high), u)

    def ball_measure(self, y, z, r):
        return self.lib.ref_ball_measure(y, z, r)

    def binmap(self, raw):
        raw = np.ascontiguousarray(raw, np.int32)
        out = np.zeros_like(raw)
        merged = self.lib.ref_binmap(raw.ctypes.data, len(raw), out.ctypes.data)
        return merged, out

    def choose_bath(self, bins, remaining, scale):
        bins = np.ascontiguousarray(bins, np.float64)
        out = C.c_double(0.0)
        binding = C.c_int(-1)
        st = self.lib.ref_choose_bath(bins.ctypes.data, len(bins), remaining, scale, C.byref(out), C.byref(binding))
        return st, out.value, binding.value

    def finish_bath(self, audit, state):
        audit = np.ascontiguousarray(audit, np.float64)
        st4 = np.ascontiguousarray(state, np.float64).copy()
        res = np.zeros(10)
        rc = self.lib.ref_finish_bath(audit.ctypes.data, len(audit), st4.ctypes.data, res.ctypes.data)
        return rc, st4, res


class RefSchedule:
    def __init__(self, host: RefHost, horizon, requested, edges):
        self.h = host
        req = np.ascontiguousarray(requested, np.float64)
        e = np.ascontiguousarray(edges, np.uint32)
        st = C.c_int(0)
        self.n = len(req)
        self.s = host.lib.ref_schedule_create(horizon, req.ctypes.data, self.n, e.ctypes.data, C.byref(st))
        self.status = st.value

    def time(self):
        return self.h.lib.ref_schedule_time(self.s)

    def end(self):
        return self.h.lib.ref_schedule_end(self.s)

    def due(self, tick):
        out = np.zeros(self.n, np.int32)
        k = self.h.lib.ref_schedule_due(self.s, tick, out.ctypes.data)
        return out[:k].tolist()

    def adapt(self, tick, groups, requested, passed):
        g = np.ascontiguousarray(groups, np.int32)
        r = np.ascontiguousarray(requested, np.float64)
        p = np.ascontiguousarray(passed, np.int32)
        return self.h.lib.ref_schedule_adapt(self.s, tick, g.ctypes.data, len(g), r.ctypes.data, p.ctypes.data)

    def advance(self, groups):
        g = np.ascontiguousarray(groups, np.int32)
        self.h.lib.ref_schedule_advance(self.s, g.ctypes.data, len(g))

    def levels(self):
        out = np.zeros(self.n, np.int32)
        self.h.lib.ref_schedule_levels(self.s, out.ctypes.data)
        return out.tolist()

    def close(self):
        if self.s:
            self.h.lib.ref_schedule_destroy(self.s)
            self.s = None
