"""Python handle over the batch C ABI (include/vh.h "batches"): an ensemble
of boost-invariant events evolved by one persistent kernel."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi as A
from .hydro import Config

EVENT_RUNNING, EVENT_FROZEN, EVENT_TAUMAX, EVENT_FAILED = 0, 1, 2, 3


def _chk(code, b=None):
    if code != A.OK:
        m = A.lib().vh_batch_last_error(b)
        raise A.VhError(code, m.decode() if m else "")


class Batch:
    def __init__(self, cfg: Config, sides_x, sides_y=None, tau0=0.6, dtau=0.02, tau_max=15.0, t_freeze_gev=0.15):
        nx = np.ascontiguousarray(sides_x, dtype=np.int32)
        ny = np.ascontiguousarray(sides_x if sides_y is None else sides_y, dtype=np.int32)
        n = len(nx)
        self.n = n
        self.nx, self.ny = nx, ny
        t0 = np.full(n, tau0) if np.isscalar(tau0) else np.ascontiguousarray(tau0, dtype=np.float64)
        dt = np.full(n, dtau) if np.isscalar(dtau) else np.ascontiguousarray(dtau, dtype=np.float64)
        tm = np.full(n, tau_max) if np.isscalar(tau_max) else np.ascontiguousarray(tau_max, dtype=np.float64)
        self.cfg = cfg
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        ip = ctypes.POINTER(ctypes.c_int)
        _chk(A.lib().vh_batch_create(ctypes.byref(self._c), n, nx.ctypes.data_as(ip), ny.ctypes.data_as(ip),
                                     A.ptr(t0), A.ptr(dt), A.ptr(tm), t_freeze_gev, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            A.lib().vh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_event(self, ev, e, ux, uy, prevu=None, pi_mode=A.PI_ZERO, pi5=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        _chk(A.lib().vh_batch_init_event(self.h, ev, A.ptr(c(e)), A.ptr(c(ux)), A.ptr(c(uy)), A.ptr(c(prevu)),
                                         pi_mode, A.ptr(c(pi5))), self.h)

    def init_glauber(self, seeds, bimp, A_nuc=208, R=6.62, aws=0.546, dmin=0.4, sigma_nn=6.4, w=0.5,
                     epeak_gev=40.0, efloor_gev=None, nthreads=0):
        if efloor_gev is None:
            from .configs import GLAUBER_FLOOR_GEV as efloor_gev
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        b = np.ascontiguousarray(bimp, dtype=np.float64)
        npart = np.zeros(self.n, dtype=np.int32)
        _chk(A.lib().vh_batch_init_glauber(self.h, s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), A.ptr(b),
                                           A_nuc, R, aws, dmin, sigma_nn, w, epeak_gev, efloor_gev, nthreads,
                                           npart.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), self.h)
        return npart

    def run(self, max_steps: int):
        sec = ctypes.c_double()
        g = ctypes.c_int()
        _chk(A.lib().vh_batch_run(self.h, max_steps, ctypes.byref(sec), ctypes.byref(g)), self.h)
        return sec.value, bool(g.value)

    def events(self):
        tau = np.zeros(self.n); steps = np.zeros(self.n, dtype=np.int32); st = np.zeros(self.n, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        _chk(A.lib().vh_batch_events(self.h, A.ptr(tau), steps.ctypes.data_as(ip), st.ctypes.data_as(ip)), self.h)
        return tau, steps, st

    def event_state(self, ev) -> np.ndarray:
        n = int((self.nx[ev] + 6) * (self.ny[ev] + 6))
        f = np.zeros((A.NFIELDS, n))
        _chk(A.lib().vh_batch_get_event_state(self.h, ev, A.ptr(f)), self.h)
        return f

    def observables(self):
        """per-event momentum anisotropy eps_p and eccentricity eps_2 of the
        current states"""
        ep, e2 = np.zeros(self.n), np.zeros(self.n)
        _chk(A.lib().vh_batch_observables(self.h, A.ptr(ep), A.ptr(e2)), self.h)
        return ep, e2

    def autotune(self, cache_path=None, probe_steps=16) -> float:
        ms = ctypes.c_double()
        _chk(A.lib().vh_batch_autotune(self.h, cache_path.encode() if cache_path else None, probe_steps,
                                       ctypes.byref(ms)), self.h)
        return ms.value

    def set_tuning(self, variant, steps_per_launch, use_graph=True):
        _chk(A.lib().vh_batch_set_tuning(self.h, variant, steps_per_launch, int(use_graph)), self.h)

    def tuning(self):
        v = [ctypes.c_int() for _ in range(5)]
        _chk(A.lib().vh_batch_get_tuning(self.h, *[ctypes.byref(x) for x in v]), self.h)
        return dict(zip(("variant", "steps_per_launch", "lines_per_tile", "blocks_per_sm", "unroll"),
                        (x.value for x in v)))
