"""The Glasma initial state on the GPU (vh_profile_cgc, vh_init_tmunu,
vh_init_prevu_tmunu) against the reference's own ginit() on one rank's
window (tests/golden/ref_cgc.npz), then a few steps from it.  The EOS is the
fixture's table of the reference's s95p parametrisation, so P(e) is its
linear interpolation: e, u and prevu (which do not depend on the EOS) are
held to rounding, pi and T^{tau mu} to the formula with the table's P and,
loosely, to the reference's values."""
import os

import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200.hydro import Config, Hydro, profile_cgc

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def table_P(tab, e):
    i = np.clip(np.searchsorted(tab[0], e, side="right") - 1, 0, tab.shape[1] - 2)
    w = (e - tab[0][i]) / (tab[0][i + 1] - tab[0][i])
    return tab[1][i] + w * (tab[1][i + 1] - tab[1][i])


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_glasma_initial_state(precision):
    g = np.load(os.path.join(HERE, "golden", "ref_cgc.npz"))
    dx, dy, dz, tau0, ts = (float(v) for v in g["consts"][:5])
    tab = g["eos_table"]
    cfg = Config(nx=60, ny=60, nz=61, boost_invariant=False, precision=precision, dx=dx, dy=dy, dz=dz, tau0=tau0,
                 dtau=ts, eos_kind=A.EOS_TABLE, eos_table=tab, etas0=1 / (4 * np.pi), etas1=0.0, hbarc=0.1973)
    peak = lambda t: 0.58 * float(g["e_at_0p4gev"]) * (t / 0.6) ** (-4.0 / 3.0)
    T = profile_cgc(60, 60, 61, False, dx, dy, dz, tau0, e_peak=peak(tau0))
    Tp = profile_cgc(60, 60, 61, False, dx, dy, dz, tau0 - ts, e_peak=peak(tau0 - ts))
    gxr, gyr = int(g["dims"][0]), int(g["dims"][1])
    c = g["cells"]
    o = (c // (gxr * gyr) * 66 + (c // gxr) % gyr) * 66 + c % gxr
    ref = g["state"]
    with Hydro(cfg) as H:
        assert H.init_tmunu(tau0, T) == 0
        assert H.init_prevu_tmunu(tau0 - ts, Tp) == 0
        s = H.get_state()[:, o]
        H.step(5)  # the evolution proceeds from it
        assert abs(H.tau - (tau0 + 5 * ts)) < 1e-12
    fp64 = precision == A.PREC_FP64
    tol = 1e-12 if fp64 else 1e-6
    assert np.max(np.abs(s[0] - ref[0]) / ref[0]) <= tol
    assert np.max(np.abs(s[1:5] - ref[1:5])) <= tol * 10
    assert np.max(np.abs(s[14:18] - ref[14:18])) <= tol * 10
    # pi with the table's P, and against the reference's s95p P
    P = table_P(tab, s[0])
    gi = np.array([1.0, -1.0, -1.0, -1.0 / tau0 ** 2])
    u = s[1:5]
    tid = (s[0] + P) * u * u - P[None, :] * gi[:, None]
    PI = -(tid[0] - tid[1] - tid[2] - tau0 ** 2 * tid[3]) / 3
    q, ab = [4, 7, 5, 6, 8], [(1, 1), (2, 2), (1, 2), (1, 3), (2, 3)]
    Tc = T[:, o]
    for m, (x, y) in enumerate(ab):
        d = (gi[x] if x == y else 0.0)
        want = Tc[q[m]] - ((s[0] + P) * u[x] * u[y] - P * d) - PI * (d - u[x] * u[y])
        assert np.max(np.abs(s[5 + m] - want) / P) <= (1e-11 if fp64 else 1e-5), m
        loose = np.max(np.abs(s[5 + m] - ref[5 + m]) / g["P"])
        print("pi component %d vs the reference (s95p P): %.1e of P" % (m, loose))
        assert loose <= 1e-4
    assert np.max(np.abs(s[10:14] - ref[10:14]) / np.abs(ref[10]).max()) <= 1e-4


def test_glasma_evolution_against_the_reference():
    """the reference's own Glasma state on one rank's window (compiled
    ginit.h, oracle/_ref/libref_ginit.so) stepped three times by the
    reference and by the FP64 GPU step, s95p as a 200,000-row table"""
    import ctypes
    from pyoracle import HERE as ORACLE_DIR
    from pyoracle import NF, RefGinit, _ptr
    if not os.path.exists(os.path.join(ORACLE_DIR, "_ref", "libref_ginit.so")):
        pytest.skip("reference GINIT build not made")
    R = RefGinit(4, 4)
    R.L.ref_ginit_step.argtypes = [ctypes.c_double, ctypes.c_double]
    f0, _, _, _ = R.run()
    te = np.geomspace(1e-2, 1e4, 200000)
    tab = np.array([R.eos(v)[:3] for v in te])
    table = np.array([te, tab[:, 0], tab[:, 1], tab[:, 2]])
    cfg = Config(nx=R.gx - 6, ny=R.gy - 6, nz=R.gz - 6, boost_invariant=False, dx=R.dx, dy=R.dy, dz=R.dz,
                 tau0=R.tau0, dtau=R.ts, eos_kind=A.EOS_TABLE, eos_table=table, etas0=1 / (4 * np.pi), etas1=0.0,
                 hbarc=R.gevfm)
    tau = R.tau0
    for _ in range(3):
        R.L.ref_ginit_step(tau, R.ts)
        tau += R.ts
    fr = np.zeros((NF, R.n))
    junk = [np.zeros(R.n) for _ in range(3)]
    R.L.ref_ginit_state(_ptr(fr), *(_ptr(a) for a in junk))
    with Hydro(cfg) as H:
        H.set_state(f0, R.tau0)
        H.step(3)
        g = H.get_state()
    idx = np.arange(R.n)
    i, j, k = idx % R.gx, (idx // R.gx) % R.gy, idx // (R.gx * R.gy)
    m = (i >= R.il) & (i < R.ir) & (j >= R.jl) & (j < R.jr) & (k >= R.kl) & (k < R.kr)
    worst = 0.0
    for grp in ((0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)):
        scale = max(np.abs(fr[q][m]).max() for q in grp)
        worst = max(worst, max(np.abs(g[q][m] - fr[q][m]).max() for q in grp) / scale)
    print("GINIT window, 3 steps: GPU vs reference %.2e (group-relative)" % worst)
    assert worst <= 1e-9
