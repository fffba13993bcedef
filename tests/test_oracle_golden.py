"""The oracle against golden fixtures made by the reference's own code.

tests/golden/ref_*.npz come from tests/golden/make_golden.py, which runs
the reference's NEWEST5 / TXYZ5 headers (compiled in oracle/_ref) on seeded
smooth states.  These CPU tests rebuild the same inputs and require the
oracle to reproduce the reference's stage terms, two full TVDRK2 steps, the
Navier-Stokes initialisation and the conserved-to-primitive residuals.
The reference itself is not needed to run them.

Tolerances: the oracle restates the reference's arithmetic; the shear
source is our covariant derivation of the same equation and the closure
A1..A5 is written in another (equivalent) form, so agreement is at the
level of a few ulps, checked at 1e-12 relative to each tensor's scale.
"""
import math
import os

import numpy as np
import pytest

from pyoracle import Oracle, OracleConfig, grid_coords, smooth_state

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
VARIANTS = {
    "milne_lbi": dict(etas0=1 / (4 * math.pi), taupi_kind=0, cartesian=False, mirror=False),
    "milne_3d": dict(etas0=1 / (4 * math.pi), taupi_kind=0, cartesian=False, mirror=False),
    "gubser": dict(etas0=0.2, taupi_kind=1, cartesian=False, mirror=True),
    "gubser_cold": dict(etas0=0.2, taupi_kind=1, cartesian=False, mirror=True, cold=True),
    "cart_3d": dict(etas0=0.01 / (4 * math.pi), taupi_kind=0, cartesian=True, mirror=False),
}
TOL = 1e-12
GROUPS = [(0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)]


def setup(variant):
    g = np.load(os.path.join(GOLD, f"ref_{variant}.npz"))
    gx, gy, gz, bi = (int(v) for v in g["dims"])
    dx, dy, dz, factor, gevfm = (float(v) for v in g["consts"])
    sc = VARIANTS[variant]
    cfg = OracleConfig(nx=gx - 6, ny=gy - 6, nz=(1 if bi else gz - 6), boost_invariant=bool(bi),
                       cartesian=sc["cartesian"], dx=dx, dy=dy, dz=dz, eos_kind=0, eos_a=factor,
                       etas0=sc["etas0"], hbarc=gevfm, taupi_kind=sc["taupi_kind"], gubser_mirror=sc["mirror"],
                       cold_plasma=sc.get("cold", False))
    x, y, z = grid_coords(gx, gy, gz, dx, dy, dz, bool(bi))
    tau, ts = float(g["tau"]), float(g["ts"])
    f = smooth_state(x, y, z, tau, ts, seed=int(g["seed"]), cartesian=sc["cartesian"])
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(tau)
    return g, O, O.get_state(), tau, ts


def scaled_err(a, b):
    s = np.max(np.abs(b))
    d = np.max(np.abs(a - b))
    return 0.0 if d == 0 else d / (s if s > 0 else 1.0)


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_stage_terms(variant):
    g, O, f, tau, ts = setup(variant)
    src, res, du = O.stage_terms(tau, ts)
    c = g["cells"]
    assert scaled_err(src[:4, c], g["src"][:4]) <= TOL      # geometric sources
    assert scaled_err(src[4:9, c], g["src"][4:9]) <= TOL    # shear sources
    assert scaled_err(res[:4, c], g["res"][:4]) <= TOL      # T^{tau mu} flux divergence
    assert scaled_err(res[4:9, c], g["res"][4:9]) <= TOL    # pi flux divergence
    assert scaled_err(du[:, c], g["du"]) <= TOL


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_two_steps(variant):
    g, O, f, tau, ts = setup(variant)
    assert O.step(tau, ts) == 0
    assert O.step(tau + ts, ts) == 0
    s = O.get_state()
    c = g["cells"]
    for grp in GROUPS:
        grp = list(grp)
        assert scaled_err(s[grp][:, c], g["step2"][grp]) <= TOL, grp
    tot = s.sum(axis=1)
    ref = g["step2_sum"]
    assert np.all(np.abs(tot - ref) <= 1e-11 * np.maximum(1.0, np.abs(ref)))


@pytest.mark.parametrize("variant", ["milne_lbi", "milne_3d", "gubser"])
def test_navier_stokes_init(variant):
    g, O, f, tau, ts = setup(variant)
    O.ns_init(tau, ts)
    s = O.get_state()
    c = g["cells"]
    assert scaled_err(s[5:10, c], g["ns"][:5]) <= TOL
    assert scaled_err(s[10:14, c], g["ns"][5:9]) <= TOL
    assert np.all(np.abs(s[5:14].sum(axis=1) - g["ns_sum"]) <= 1e-11 * np.maximum(1.0, np.abs(g["ns_sum"])))


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_con2prim_residuals(variant):
    g, O, f, tau, ts = setup(variant)
    for x, p, y, J in zip(g["res_x"], g["res_p"], g["res_y"], g["res_J"]):
        yo, Jo = O.residual(x, p)
        scale = np.max(np.abs(p[:4])) * max(1.0, np.max(np.abs(x)))
        assert np.max(np.abs(yo - y)) <= 1e-13 * scale
        assert np.max(np.abs(Jo - J)) <= 1e-13 * max(1.0, np.max(np.abs(J)))


def test_cartesian_shock_tube():
    """The reference's own Cartesian scenario: the oracle runs the shock tube
    20 steps and reproduces the reference's state at every interior cell"""
    from helpers import shock_tube_fixture
    g, cfg, f = shock_tube_fixture()
    O = Oracle(cfg)
    O.set_state(f)
    t = 0.0
    for _ in range(int(g["steps"])):
        assert O.step(t, float(g["ts"])) == 0
        t += float(g["ts"])
    s = O.get_state()
    c = g["cells"]
    for grp in GROUPS:
        grp = [q for q in grp if q < 14]
        if grp:
            assert scaled_err(s[grp][:, c], g["state"][grp]) <= TOL, grp
    assert np.allclose(s.sum(axis=1)[:14], g["state_sum"][:14], rtol=1e-12, atol=1e-9)


def test_navier_stokes_shear_ten_components():
    """NEWEST10's CalcNS (ten components of 2 eta sigma^{mu nu} as expanded
    polynomials): the oracle's projector form at the reference's own
    velocity derivatives, with u^eta and d_eta u^mu nonzero, and the
    oracle's velocity derivatives against the reference's"""
    g = np.load(os.path.join(GOLD, "ref_ns10_lbi.npz"))
    gx, gy, gz, _ = (int(v) for v in g["dims"])
    dx, dy, factor = (float(v) for v in g["consts"])
    tau, ts = float(g["tau"]), float(g["ts"])
    cfg = OracleConfig(nx=gx - 6, ny=gy - 6, nz=1, boost_invariant=True, cartesian=False, dx=dx, dy=dy, dz=0.1,
                       eos_kind=0, eos_a=factor, etas0=1 / (4 * math.pi), hbarc=0.1973, taupi_kind=0)
    x, y, z = grid_coords(gx, gy, gz, dx, dy, 0.1, True)
    f = smooth_state(x, y, z, tau, ts, seed=int(g["seed"]))
    assert np.abs(f[4]).max() > 0.01  # u^eta is exercised
    O = Oracle(cfg)
    O.set_state(f)
    cells, ns, du = g["cells"], g["ns"], g["du"]
    assert np.all(ns[10] == 0)  # no bulk viscosity in the build
    mine = np.array([O.ns_pi10_cell(tau, f[0, c], f[1:5, c], du[:, a]) for a, c in enumerate(cells)]).T
    for q in range(10):
        assert scaled_err(mine[q], ns[q]) <= TOL, q
    # the step's velocity derivatives (d_tau from prevu, WENO in x and y)
    grid = O.ns_pi10(tau, ts)
    _, _, odu = O.stage_terms(tau, ts)
    for q in range(16):
        if q % 4 != 3:
            assert scaled_err(odu[q, cells], du[q]) <= TOL, q
    # with d_eta u = 0 (what a boost-invariant grid has) the grid path equals
    # the pointwise one
    du0 = du.copy()
    du0[3::4] = 0
    again = np.array([O.ns_pi10_cell(tau, f[0, c], f[1:5, c], du0[:, a]) for a, c in enumerate(cells)]).T
    assert np.array_equal(grid[:, cells], again)


def bjorken_oracle(g):
    gx, gy, gz, _ = (int(v) for v in g["dims"])
    dx, dy, dz, factor, gevfm = (float(v) for v in g["consts"])
    cfg = OracleConfig(nx=gx - 6, ny=gy - 6, nz=1, boost_invariant=True, dx=dx, dy=dy, dz=dz, eos_kind=0,
                       eos_a=factor, etas0=0.2, etas1=0.0, hbarc=gevfm, taupi_kind=2, taupi_const=0.01)
    f = np.zeros((18, gx * gy))
    f[0] = 30.0 / gevfm
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(float(g["tau0"]))
    return O


def test_bjorken_scenario():
    """The reference's Bjorken scenario (uniform fluid at rest in Milne
    coordinates, eta/s = 0.2, tau_pi = 0.01 fm/c) to tau = 10 fm/c: the
    oracle's centre temperature after every step is the reference's, and it
    follows first-order viscous Bjorken flow,
    T = T0 (tau0/tau)^(1/3) [1 + 2 (eta/s) (1 - (tau0/tau)^(2/3)) / (3 tau0 T0)],
    to 0.2 % (the viscous heating itself is 10 % at tau = 10)"""
    g = np.load(os.path.join(GOLD, "ref_bjorken.npz"))
    O = bjorken_oracle(g)
    c, ts = int(g["centre"]), float(g["ts"])
    tau, temps = float(g["tau0"]), []
    for _ in range(int(g["steps"])):
        assert O.step(tau, ts) == 0
        tau += ts
        temps.append(O.eos(O.get_state()[0, c])[2])
    temps = np.array(temps)
    assert np.max(np.abs(temps - g["temp"]) / g["temp"]) <= TOL
    assert scaled_err(O.get_state()[:, c], g["final"]) <= TOL
    t0, T0 = float(g["tau0"]), (30.0 / float(g["consts"][4]) / float(g["consts"][3])) ** 0.25
    taus = t0 + ts * np.arange(1, len(temps) + 1)
    first_order = T0 * (t0 / taus) ** (1 / 3) * (1 + 2 * 0.2 * (1 - (t0 / taus) ** (2 / 3)) / (3 * t0 * T0))
    assert np.max(np.abs(temps / first_order - 1)) <= 2e-3
    assert temps[-1] / (T0 * (t0 / taus[-1]) ** (1 / 3)) - 1 > 0.09


def test_cartesian_bjorken_block():
    """The reference's Cartesian Bjorken block (TXYZ5, -DBJORKEN): a uniform
    fluid at rest in (t, x, y, z) is an equilibrium, and the compiled
    reference keeps it bitwise for 100 steps; so does the oracle"""
    g = np.load(os.path.join(GOLD, "ref_cart_bjorken.npz"))
    gx, gy, gz, _ = (int(v) for v in g["dims"])
    dx, dy, dz, factor, gevfm = (float(v) for v in g["consts"])
    cfg = OracleConfig(nx=gx - 6, ny=gy - 6, nz=gz - 6, boost_invariant=False, cartesian=True, dx=dx, dy=dy, dz=dz,
                       eos_kind=0, eos_a=factor, etas0=0.2, etas1=0.0, hbarc=gevfm, taupi_kind=2, taupi_const=0.01)
    f = np.zeros((18, gx * gy * gz))
    f[0] = 30.0 / gevfm
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(float(g["t0"]))
    f = O.get_state()
    assert np.array_equal(f[:, int(g["centre"])], g["initial"])
    t = float(g["t0"])
    for _ in range(int(g["steps"])):
        assert O.step(t, float(g["ts"])) == 0
        t += float(g["ts"])
    s = O.get_state()
    assert np.all(g["max_change"] == 0) and np.array_equal(s, f)
    assert np.array_equal(s[:, int(g["centre"])], g["final"])
