"""ctypes binding of the C ABI in include/vh.h (libvh.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback
for the step.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvh.so")

NFIELDS = 18
NGHOST = 3
STATIC_MAX_CELLS = 61680  # VH_STATIC_MAX_CELLS

# vh_status
OK, E_ARG, E_CUDA, E_ROOTFIND, E_CAUSALITY, E_NEG_ENERGY, E_TIMEOUT, E_STATE, E_NOMEM, E_UNSUPPORTED = range(10)
STATUS_NAMES = {0: "VH_OK", 1: "VH_E_ARG", 2: "VH_E_CUDA", 3: "VH_E_ROOTFIND", 4: "VH_E_CAUSALITY",
                5: "VH_E_NEG_ENERGY", 6: "VH_E_TIMEOUT", 7: "VH_E_STATE", 8: "VH_E_NOMEM", 9: "VH_E_UNSUPPORTED"}
COORD_MILNE, COORD_CARTESIAN = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
RECON_WENO5, RECON_MINMOD = 0, 1
EOS_CONFORMAL, EOS_TABLE = 0, 1
TAUPI_15_ETA_OVER_P, TAUPI_5_ETA_OVER_EPP, TAUPI_CONST = 0, 1, 2
PI_GIVEN, PI_ZERO, PI_NS = 0, 1, 2
WRITE_XY, WRITE_FULL, WRITE_XY17, WRITE_FULL17, WRITE_NS_XY = 0, 1, 2, 3, 4

_dp = ctypes.POINTER(ctypes.c_double)


class VhConfig(ctypes.Structure):
    _fields_ = [
        ("coords", ctypes.c_int), ("precision", ctypes.c_int), ("recon", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("boost_invariant", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("tau0", ctypes.c_double), ("dtau", ctypes.c_double),
        ("eos_kind", ctypes.c_int), ("eos_a", ctypes.c_double), ("eos_n", ctypes.c_int),
        ("eos_e", _dp), ("eos_p", _dp), ("eos_cs2", _dp), ("eos_t", _dp),
        ("etas0", ctypes.c_double), ("etas1", ctypes.c_double), ("etas_tc", ctypes.c_double),
        ("hbarc", ctypes.c_double),
        ("taupi_kind", ctypes.c_int), ("gubser_mirror", ctypes.c_int), ("minmod_theta", ctypes.c_double),
        ("taupi_const", ctypes.c_double), ("cold_plasma", ctypes.c_int),
    ]


# (name, restype, argtypes) of every entry point declared in include/vh.h
SIGNATURES = [
    ("vh_create", ctypes.c_int, [ctypes.POINTER(VhConfig), ctypes.POINTER(ctypes.c_void_p)]),
    ("vh_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("vh_set_stream", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("vh_dims", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int)]),
    ("vh_set_state", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_double]),
    ("vh_get_state", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_set_state_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]),
    ("vh_get_state_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("vh_get_primitive", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    ("vh_landau_match", ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_double, ctypes.c_int, _dp, _dp,
                                       ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_init_tmunu", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_init_profile", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, _dp]),
    ("vh_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("vh_get_time", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_max_temperature", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_conservation_sums", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_cfl", ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    ("vh_write", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]),
    ("vh_debug_stage_terms", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp]),
    ("vh_time_kernels", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    ("vh_last_iterations", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_sweep_uses_tma", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    ("vh_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("vh_step_static", ctypes.c_int, [ctypes.POINTER(VhConfig), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_void_p]),
    ("vh_eos_table_synthetic", ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, _dp, _dp, _dp, _dp]),
    ("vh_profile_gubser", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]),
    ("vh_profile_glauber", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_uint64, _dp,
                                          ctypes.POINTER(ctypes.c_int)]),
    ("vh_batch_create", ctypes.c_int, [ctypes.POINTER(VhConfig), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    ("vh_batch_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("vh_batch_reset", ctypes.c_int, [ctypes.c_void_p]),
    ("vh_batch_init_event", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, _dp]),
    ("vh_batch_init_glauber", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), _dp, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_int)]),
    ("vh_batch_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]),
    ("vh_batch_events", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    ("vh_batch_get_event_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    ("vh_batch_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, _dp]),
    ("vh_batch_set_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("vh_batch_get_tuning", ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 5),
    ("vh_batch_observables", ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    ("vh_batch_barrier_selftest", ctypes.c_int, [ctypes.c_int, _dp]),
    ("vh_get_ns_pi", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_get_conserved", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_profile_gubser_cold", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, _dp, _dp, _dp, _dp, _dp]),
    ("vh_profile_gubser_is", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            _dp, _dp, _dp, _dp, _dp]),
    ("vh_freezeout_2d", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _dp, _dp, _dp, _dp, ctypes.c_double, _dp, ctypes.c_longlong,
                                       ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_freezeout_3d", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp,
                                       ctypes.c_double, _dp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_cooper_frye_2d", ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp,
                                         ctypes.c_int, _dp, ctypes.c_int, _dp]),
    ("vh_cooper_frye_3d", ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp]),
    ("vh_freezeout_2d_device", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                              ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]),
    ("vh_freezeout_3d_device", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]),
    ("vh_freezeout_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong,
                                         ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_cooper_frye_2d_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                                ctypes.c_void_p]),
    ("vh_cooper_frye_3d_device", ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int, _dp,
                                                ctypes.c_int, _dp, ctypes.c_void_p]),
    ("vh_init_prevu_tmunu", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    ("vh_profile_cgc", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, _dp]),
    ("vh_save_checkpoint", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("vh_load_checkpoint", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _dp]),
    ("vh_batch_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("vh_read_ideal_profile", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                             ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("vh_eps_p", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("vh_adjoint_eps_p", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("vh_adjoint_phase_times", ctypes.c_int, [ctypes.c_void_p, _dp]),
]

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded libvh.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m viral_b200.build` "
                               "(the step has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class VhError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(code: int, handle=None):
    if code != OK:
        m = lib().vh_last_error(handle)
        raise VhError(code, m.decode() if m else "")


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "arrays must be C-contiguous float64"
    return a.ctypes.data_as(_dp)
