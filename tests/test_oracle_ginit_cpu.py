"""The oracle against the reference evolving its own realistic scenario: the
GINIT block (NEWEST5/ginit.h initial state, s95p EOS, tau0 = 0.1 fm/c,
ts = 0.002) on one rank's 3+1D window, three TVDRK2 steps of the compiled
reference (oracle/_ref/libref_ginit.so, oracle/ref_ginit.cpp) against three
oracle steps from the same state.  The oracle takes the s95p EOS as a table
of 200,000 rows sampled from the reference's functions (linear
interpolation error ~1e-9).  Needs the reference build (skipped where it
was not made)."""
import ctypes
import os

import numpy as np
import pytest

from pyoracle import HERE as ORACLE_DIR
from pyoracle import NF, Oracle, OracleConfig, RefGinit, _ptr

LIB = os.path.join(ORACLE_DIR, "_ref", "libref_ginit.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference GINIT build not made")
def test_oracle_evolves_the_glasma_state_like_the_reference():
    R = RefGinit(4, 4)
    R.L.ref_ginit_step.argtypes = [ctypes.c_double, ctypes.c_double]
    f0, _, _, _ = R.run()
    te = np.geomspace(1e-2, 1e4, 200000)
    tab = np.array([R.eos(v)[:3] for v in te])
    table = np.array([te, tab[:, 0], tab[:, 1], tab[:, 2]])
    cfg = OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=R.gz - 6, boost_invariant=False, cartesian=False, dx=R.dx,
                       dy=R.dy, dz=R.dz, eos_kind=1, eos_table=table, etas0=1 / (4 * np.pi), etas1=0.0,
                       hbarc=R.gevfm, taupi_kind=0)
    O = Oracle(cfg)
    O.set_state(f0)
    tau = R.tau0
    for _ in range(3):
        R.L.ref_ginit_step(tau, R.ts)
        assert O.step(tau, R.ts) == 0
        tau += R.ts
    fr = np.zeros((NF, R.n))
    junk = [np.zeros(R.n) for _ in range(3)]
    R.L.ref_ginit_state(_ptr(fr), *(_ptr(a) for a in junk))
    fo = O.get_state()
    idx = np.arange(R.n)
    i, j, k = idx % R.gx, (idx // R.gx) % R.gy, idx // (R.gx * R.gy)
    m = (i >= R.il) & (i < R.ir) & (j >= R.jl) & (j < R.jr) & (k >= R.kl) & (k < R.kr)
    worst = 0.0
    for grp in ((0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)):
        scale = max(np.abs(fr[q][m]).max() for q in grp)
        err = max(np.abs(fo[q][m] - fr[q][m]).max() for q in grp) / scale
        worst = max(worst, err)
    print("GINIT window, 3 steps: oracle vs reference %.2e (group-relative)" % worst)
    assert worst <= 1e-9
