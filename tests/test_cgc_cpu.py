"""The Glasma (optical-Glauber CGC) initial state against the reference's own
ginit() (NEWEST5/ginit.h compiled in oracle/_ref; fixture
tests/golden/ref_cgc.npz, made by tests/golden/make_golden.py): the tensor
of vh_profile_cgc (host code), Landau-matched by the same function the GPU
kernel runs (the check library's CPU build), gives the reference's e and u
at tau0 and its prevu at tau0 - ts; pi from the reference's formula
(ginit.h:955-989) with the reference's own P(e) gives its pi.  The fixture
is one rank's window (x, y in [-3.3, 0.2] fm, eta in [-3.3, 3.3]) of the
reference's 300 x 300 x 61 grid; our grid of 60 x 60 x 61 cells starts at
the same corner."""
import ctypes
import os

import numpy as np
import pytest

from viral_b200 import build
from viral_b200.hydro import profile_cgc

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "ref_cgc.npz"))


@pytest.fixture(scope="module")
def ours(gold):
    dx, dy, dz, tau0, ts = (float(v) for v in gold["consts"][:5])
    e06 = float(gold["e_at_0p4gev"])
    peak = lambda t: 0.58 * e06 * (t / 0.6) ** (-4.0 / 3.0)
    T = profile_cgc(60, 60, 61, False, dx, dy, dz, tau0, e_peak=peak(tau0))
    Tp = profile_cgc(60, 60, 61, False, dx, dy, dz, tau0 - ts, e_peak=peak(tau0 - ts))
    return T, Tp


def our_index(gold):
    gxr, gyr = int(gold["dims"][0]), int(gold["dims"][1])
    c = gold["cells"]
    i, j, k = c % gxr, (c // gxr) % gyr, c // (gxr * gyr)
    return (k * 66 + j) * 66 + i


def landau(T10, tau):
    L = ctypes.CDLL(build.build_check())
    L.vhc_landau.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp, _dp]
    e = ctypes.c_double()
    u = np.zeros(4)
    t = np.ascontiguousarray(T10, dtype=np.float64)
    assert L.vhc_landau(t.ctypes.data_as(_dp), tau, 0, ctypes.byref(e), u.ctypes.data_as(_dp)) == 1
    return e.value, u


def test_grid_matches_the_reference_window(gold):
    gxr, gyr = int(gold["dims"][0]), int(gold["dims"][1])
    c = gold["cells"]
    i, j, k = c % gxr, (c // gxr) % gyr, c // (gxr * gyr)
    assert np.allclose(gold["x"], -3.0 + (i - 3) * 0.1, atol=1e-12)
    assert np.allclose(gold["y"], -3.0 + (j - 3) * 0.1, atol=1e-12)
    assert np.allclose(gold["eta"], -3.0 + (k - 3) * 0.1, atol=1e-12)
    assert np.abs(gold["eta"]).max() > 2.5  # the Gaussian eta tails are sampled


def test_energy_density_velocity_and_prevu(gold, ours):
    T, Tp = ours
    tau0, ts = float(gold["consts"][3]), float(gold["consts"][4])
    s = gold["state"]
    errs = []
    for a, o in enumerate(our_index(gold)):
        e, u = landau(T[:, o], tau0)
        _, up = landau(Tp[:, o], tau0 - ts)
        errs.append((abs(e - s[0, a]) / s[0, a], np.max(np.abs(u - s[1:5, a])), np.max(np.abs(up - s[14:18, a]))))
    errs = np.array(errs)
    print("e, u, prevu max errors:", errs.max(axis=0))
    assert errs[:, 0].max() <= 1e-12 and errs[:, 1].max() <= 1e-12 and errs[:, 2].max() <= 1e-12
    assert np.abs(s[4]).max() > 0.01  # longitudinal flow is present


def test_shear_tensor_formula(gold, ours):
    """pi^{ab} = T^{ab} - T_id^{ab} - PI (g^{ab} - u^a u^b), PI = -(e - 3P)/3"""
    T, _ = ours
    tau0 = float(gold["consts"][3])
    s, P = gold["state"], gold["P"]
    q, ab = [4, 7, 5, 6, 8], [(1, 1), (2, 2), (1, 2), (1, 3), (2, 3)]
    gi = np.array([1.0, -1.0, -1.0, -1.0 / tau0 ** 2])
    worst = 0.0
    for a, o in enumerate(our_index(gold)):
        e, u = landau(T[:, o], tau0)
        tid = (e + P[a]) * u * u - P[a] * gi
        PI = -(tid[0] - tid[1] - tid[2] - tau0 ** 2 * tid[3]) / 3
        for m, (x, y) in enumerate(ab):
            idl = (e + P[a]) * u[x] * u[y] - (P[a] * gi[x] if x == y else 0.0)
            pim = PI * ((gi[x] if x == y else 0.0) - u[x] * u[y])
            worst = max(worst, abs(T[q[m], o] - idl - pim - s[5 + m, a]) / P[a])
    print("pi: max |ours - reference| / P = %.2e" % worst)
    assert worst <= 1e-11
