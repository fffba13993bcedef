"""vh_step_static, the step that allocates nothing, against vh_step.

vh_step_static serves callers that must not call cudaMalloc where they
advance the fluid: a code whose device memory belongs to another framework's
pool allocator, where an allocation behind the pool's back would break the
budget it was given.  They own the state and lend it to the call; the step's
scratch sits in a static device array inside the library.  This file runs
last so that a failure here leaves every other test already run.

Two calls in a row on the same state must match two vh_step calls on a
handle, to the FP64 tolerance of the other GPU tests (1e-12 of each tensor
group's scale), for
boost-invariant and 3+1D Milne grids, a Cartesian grid, both EOS kinds and a
grid of exactly the largest size; the first call's leftovers in the shared
scratch must not leak into the second, and the second call must leave the
device's free memory unchanged.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from helpers import smooth_inputs  # noqa: E402
from viral_b200 import _abi as A  # noqa: E402
from viral_b200 import configs as C  # noqa: E402
from viral_b200.hydro import Config, Hydro  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-12
# fields compared on the scale of their tensor group (as the parity tests):
# e; u^mu; pi^{mu nu}; T^{tau mu}; prevu
GROUPS = [(0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)]
MAX_CELLS = 61680  # VH_STATIC_MAX_CELLS in include/vh.h


def _static(cfg, dev, eos_dev, tau, n, stream):
    c = cfg.to_c()
    return A.lib().vh_step_static(ctypes.byref(c), ctypes.c_void_p(dev.data_ptr()),
                                  ctypes.c_void_p(eos_dev.data_ptr()) if eos_dev is not None else None,
                                  tau, n, ctypes.c_void_p(stream))


def _run_pair(cfg, f0, tau0, steps=(3, 2)):
    """vh_step on a handle and vh_step_static on a device copy of the same
    18-field state, `steps` steps per call; also the device's free memory
    before and after the second static call"""
    import torch
    with Hydro(cfg) as H:
        H.set_state(f0, tau0)
        ref = []
        for n in steps:
            H.step(n)
            ref.append(H.get_state())
    dev = torch.from_numpy(np.ascontiguousarray(f0).reshape(-1).copy()).cuda()
    eos_dev = None
    if cfg.eos_kind == A.EOS_TABLE:
        eos_dev = torch.from_numpy(np.ascontiguousarray(cfg.eos_table).reshape(-1).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    tau = tau0
    got, free = [], []
    for q, n in enumerate(steps):
        if q == len(steps) - 1:
            free.append(torch.cuda.mem_get_info()[0])
        rc = _static(cfg, dev, eos_dev, tau, n, stream)
        assert rc == A.OK, A.STATUS_NAMES.get(rc, rc)
        if q == len(steps) - 1:
            free.append(torch.cuda.mem_get_info()[0])
        for _ in range(n):  # the time advances by repeated addition, as in the library
            tau += cfg.dtau
        got.append(dev.cpu().numpy().reshape(A.NFIELDS, -1).copy())
    return ref, got, free


def _from_inputs(cfg, inp):
    with C.make_hydro(cfg, inp) as H:
        return H.get_state(), H.tau


def _case(which):
    if which == "gubser":
        cfg = C.gubser_config(nx=65, ny=65)
        return (cfg, *_from_inputs(cfg, C.gubser_inputs(cfg)))
    if which == "glauber_table":
        cfg = C.glauber_config(nx=96, ny=96, boost_invariant=True)
        return (cfg, *_from_inputs(cfg, C.glauber_inputs(cfg, b=5.0, seed=4)))
    if which == "glauber_3d_table":
        cfg = C.glauber_config(nx=24, ny=22, nz=12)
        return (cfg, *_from_inputs(cfg, C.glauber_inputs(cfg, b=5.0, seed=2)))
    if which == "cartesian_3d":
        cfg = Config(nx=20, ny=18, nz=12, boost_invariant=False, coords=A.COORD_CARTESIAN, dx=0.1, dy=0.1, dz=0.1,
                     tau0=1.0, dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=13.899692864867510, etas0=1 / (4 * np.pi))
        return cfg, smooth_inputs(cfg, cfg.tau0, seed=5), cfg.tau0
    if which == "largest_grid":
        # 240 x 257 ghost-inclusive cells: exactly VH_STATIC_MAX_CELLS
        cfg = C.glauber_config(nx=234, ny=251, boost_invariant=True)
        return (cfg, *_from_inputs(cfg, C.glauber_inputs(cfg, b=3.0, seed=1)))
    raise ValueError(which)


@pytest.mark.parametrize("which", ["gubser", "glauber_table", "glauber_3d_table", "cartesian_3d", "largest_grid"])
def test_static_step_matches_handle_step_twice(which):
    cfg, f0, tau0 = _case(which)
    gx, gy, gz = cfg.gdims()
    assert gx * gy * gz <= MAX_CELLS
    ref, got, free = _run_pair(cfg, f0, tau0)
    for r, g in zip(ref, got):
        for grp in GROUPS:
            scale = max(float(np.max(np.abs(r[q]))) for q in grp)
            for q in grp:
                assert np.max(np.abs(g[q] - r[q])) <= TOL * scale, f"field {q}"
    assert free[0] == free[1], f"device free memory changed by {free[0] - free[1]} bytes"


def test_static_step_rejects_bad_arguments():
    """every call below is refused on the host before anything is launched;
    the buffers are sized for the grid all the same (zero state, the real
    EOS table), so a check that let one through could not reach outside them"""
    import torch

    def rc(cfg, tau=0.6):
        gx, gy, gz = cfg.gdims()
        buf = torch.zeros(A.NFIELDS * gx * gy * gz, dtype=torch.float64, device="cuda")
        eos = None
        if cfg.eos_kind == A.EOS_TABLE:
            eos = torch.from_numpy(np.ascontiguousarray(cfg.eos_table).reshape(-1).copy()).cuda()
        c = cfg.to_c()
        r = A.lib().vh_step_static(ctypes.byref(c), ctypes.c_void_p(buf.data_ptr()),
                                   ctypes.c_void_p(eos.data_ptr()) if eos is not None else None, tau, 1, None)
        torch.cuda.synchronize()
        return r

    # 87 x 709 = 61683 ghost-inclusive cells, the smallest grid above the limit
    assert rc(C.glauber_config(nx=81, ny=703, boost_invariant=True)) == A.E_ARG
    assert rc(C.glauber_config(nx=161, ny=161, nz=41)) == A.E_ARG
    assert rc(C.gubser_config(nx=33, ny=33, precision=A.PREC_MIXED), tau=1.0) == A.E_ARG
    # Milne sources divide by tau
    g = C.gubser_config(nx=33, ny=33)
    assert rc(g, tau=0.0) == A.E_ARG
    assert rc(g, tau=-1.0) == A.E_ARG
    # the table lookup needs increasing energy densities
    t = C.glauber_config(nx=20, ny=20, boost_invariant=True)
    bad = np.array(t.eos_table, copy=True)
    bad[0, 10] = bad[0, 9]
    t.eos_table = bad
    assert rc(t) == A.E_ARG
