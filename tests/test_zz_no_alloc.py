"""vh_step_static, the step that allocates nothing, against vh_step.

vh_step_static serves callers that must not call cudaMalloc where they
advance the fluid: a code whose device memory belongs to another framework's
pool, or one recording its launches into a CUDA stream capture.  They own
the state and lend it to the call; the step's scratch sits in a static
device array inside the library.  This file runs last so that a failure here
leaves every other test already run.

Two calls in a row on the same state must match two vh_step calls on a
handle, to the FP64 tolerance of the other GPU tests (1e-12 relative), for
both EOS kinds; the first call's leftovers in the shared scratch must not
leak into the second.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from viral_b200 import _abi as A
from viral_b200 import configs as C

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _run_pair(cfg, inp, steps=(3, 2)):
    import torch
    with C.make_hydro(cfg, inp) as H:
        f0 = H.get_state()
        tau0 = H.tau
        ref = []
        for n in steps:
            H.step(n)
            ref.append(H.get_state())
    dev = torch.from_numpy(f0.reshape(-1).copy()).cuda()
    eos_dev = None
    if cfg.eos_kind == A.EOS_TABLE:
        eos_dev = torch.from_numpy(np.ascontiguousarray(cfg.eos_table).reshape(-1).copy()).cuda()
    c = cfg.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    tau = tau0
    got = []
    for n in steps:
        rc = A.lib().vh_step_static(ctypes.byref(c), ctypes.c_void_p(dev.data_ptr()),
                                    ctypes.c_void_p(eos_dev.data_ptr()) if eos_dev is not None else None,
                                    tau, n, ctypes.c_void_p(stream))
        assert rc == A.OK, A.STATUS_NAMES.get(rc, rc)
        tau += n * cfg.dtau
        got.append(dev.cpu().numpy().reshape(A.NFIELDS, -1).copy())
    return ref, got


@pytest.mark.parametrize("which", ["gubser", "glauber_table"])
def test_static_step_matches_handle_step_twice(which):
    if which == "gubser":
        cfg = C.gubser_config(nx=65, ny=65)
        inp = C.gubser_inputs(cfg)
    else:
        cfg = C.glauber_config(nx=96, ny=96, boost_invariant=True)
        inp = C.glauber_inputs(cfg, b=5.0, seed=4)
    ref, got = _run_pair(cfg, inp)
    for r, g in zip(ref, got):
        for q in range(A.NFIELDS):
            assert rel_err(g[q], r[q]) <= TOL, f"field {q}"


def test_static_step_rejects_oversized_and_mixed():
    import torch
    big = C.glauber_config(nx=161, ny=161, nz=41)
    c = big.to_c()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = A.lib().vh_step_static(ctypes.byref(c), ctypes.c_void_p(buf.data_ptr()), None, 0.6, 1, None)
    assert rc == A.E_ARG
    mixed = C.gubser_config(nx=33, ny=33, precision=A.PREC_MIXED).to_c()
    rc = A.lib().vh_step_static(ctypes.byref(mixed), ctypes.c_void_p(buf.data_ptr()), None, 1.0, 1, None)
    assert rc == A.E_ARG
