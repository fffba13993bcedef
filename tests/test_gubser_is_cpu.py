"""The semi-analytic Israel-Stewart Gubser flow, pinned to the reference's
own data, and the product's generator of its initial state.

The reference's viscous Gubser test initialises from a table
(NEWEST5/init.h:419-459); the table it opens is not shipped, but
NEWEST5/init/tempbin-8.7z holds another one (326 x 326 cells of 0.05 fm at
tau0 = 1 fm/c, q = 1/fm).  Its cells (tests/golden/ref_gubser_is_table.npz,
made by tests/golden/make_golden.py) are the solution of the de Sitter-time
equations in oracle/gubser_is.py with T^ = 1.2, P = 0 at rho = 0 and
eta/s = 0.2: the oracle reproduces them to the table's own digits (1.3e-7
in T, 5e-7 of the largest pi component), and so does vh_profile_gubser_is,
whose RK4 is independent of the oracle's SciPy integrator.  The oracle's
step, started from that state, follows the ODE."""
import math
import os

import numpy as np
import pytest

from gubser_is import GubserIS, milne_fields, rho_of
from helpers import canonical_state, interior_mask, oracle_config
from pyoracle import Oracle
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import profile_gubser_is

HERE = os.path.dirname(os.path.abspath(__file__))
REF_A = 3 * 42.25 * math.pi ** 2 / 90  # FACTOR of the reference's blocks (DOF = 42.25)
PI_COLS = {"tt": 1, "tx": 2, "ty": 3, "xx": 4, "xy": 5, "yy": 6, "ee": 7}


def _table():
    g = np.load(os.path.join(HERE, "golden", "ref_gubser_is_table.npz"))
    n = int(g["dims"][0]) - 6
    x0 = -(n // 2) * 0.05
    return g, n, x0 + (g["i"] - 3) * 0.05, x0 + (g["j"] - 3) * 0.05


def test_ode_reproduces_the_reference_table():
    g, _, X, Y = _table()
    v = g["values"]
    T, e, u, pi = milne_fields(GubserIS(1.2, 0.0, 0.2), 1.0, X, Y, REF_A)
    assert np.max(np.abs(T - v[:, 0]) / v[:, 0]) < 3e-7
    for nm, q in PI_COLS.items():
        assert np.max(np.abs(pi[nm] - v[:, q])) < 1e-6 * np.max(np.abs(v[:, q])), nm


def test_generator_reproduces_the_reference_table():
    g, n, _, _ = _table()
    hbarc = 0.19733
    e, ux, uy, pi5, pu = profile_gubser_is(n, n, 0.05, 0.05, 1.0, 1.0, 0.001, 1.2 * hbarc, 0.0, 0.2, REF_A, hbarc)
    c = g["j"] * (n + 6) + g["i"]
    v = g["values"]
    T = (e[c] / REF_A) ** 0.25
    assert np.max(np.abs(T - v[:, 0]) / v[:, 0]) < 3e-7
    for row, nm in ((0, "xx"), (1, "yy"), (2, "xy")):
        q = PI_COLS[nm]
        assert np.max(np.abs(pi5[row][c] - v[:, q])) < 1e-6 * np.max(np.abs(v[:, q])), nm
    assert np.all(pi5[3] == 0) and np.all(pi5[4] == 0)


@pytest.mark.parametrize("t0_gev", [0.6, 0.236796])
def test_generator_matches_the_ode(t0_gev):
    """c0's grid (129 x 129, 0.1 fm): the product's RK4 against the oracle's
    DOP853, every cell, and prevu the Gubser velocity at tau0 - dtau"""
    cfg = C.gubser_config()
    n = cfg.nx
    e, ux, uy, pi5, pu = profile_gubser_is(n, n, cfg.dx, cfg.dy, 1.0, 1.0, cfg.dtau, t0_gev, 0.0, 0.2, cfg.eos_a,
                                           cfg.hbarc)
    gx = n + 6
    idx = np.arange(gx * gx)
    x0 = -(n // 2) * cfg.dx
    X, Y = x0 + (idx % gx - 3) * cfg.dx, x0 + (idx // gx - 3) * cfg.dx
    S = GubserIS(t0_gev / cfg.hbarc, 0.0, 0.2)
    T, eo, u, pi = milne_fields(S, 1.0, X, Y, cfg.eos_a)
    assert np.max(np.abs(e - eo) / eo) < 1e-9
    assert np.max(np.abs(ux - u[1])) < 1e-12 and np.max(np.abs(uy - u[2])) < 1e-12
    w = (4 / 3) * eo
    for row, nm in ((0, "xx"), (1, "yy"), (2, "xy")):
        assert np.max(np.abs(pi5[row] - pi[nm]) / w) < 1e-9, nm
    _, _, up, _ = milne_fields(S, 1.0 - cfg.dtau, X, Y, cfg.eos_a)
    assert np.max(np.abs(pu - up)) < 1e-12


def test_oracle_step_follows_the_ode():
    """The oracle's step (the reference's arithmetic) from the semi-analytic
    state, 61 x 61 cells of 0.1 fm, 40 steps to tau = 1.4 fm/c: T and the
    shear ratio P = tau^2 pi^{eta eta}/(e+P) within 2 fm of the centre agree
    with the ODE to the scheme's discretisation error"""
    t0 = 1.2 * 0.19733
    cfg = C.gubser_config(nx=61, ny=61)
    n = cfg.nx
    e, ux, uy, pi5, pu = profile_gubser_is(n, n, cfg.dx, cfg.dy, 1.0, cfg.tau0, cfg.dtau, t0, 0.0, 0.2, cfg.eos_a,
                                           cfg.hbarc)
    inp = dict(tau=cfg.tau0, e=e, ux=ux, uy=uy, ueta=None, prevu=pu, pi_mode=A.PI_GIVEN)
    f = canonical_state(cfg, inp)
    f[5:10] = pi5
    O = Oracle(oracle_config(cfg))
    O.set_state(f)
    O.fill_tmunu(cfg.tau0)
    tau = cfg.tau0
    for _ in range(40):
        assert O.step(tau, cfg.dtau) == 0
        tau += cfg.dtau
    st = O.get_state()
    gx = n + 6
    idx = np.arange(gx * gx)
    x0 = -(n // 2) * cfg.dx
    X, Y = x0 + (idx % gx - 3) * cfg.dx, x0 + (idx // gx - 3) * cfg.dx
    m = interior_mask(cfg) & (np.hypot(X, Y) < 2.0)
    T, eo, u, pi = milne_fields(GubserIS(t0 / cfg.hbarc, 0.0, 0.2), tau, X, Y, cfg.eos_a)
    Tn = (st[0] / cfg.eos_a) ** 0.25
    assert np.max(np.abs(Tn[m] - T[m]) / T[m]) < 1e-3
    u0, u1, u2 = st[1], st[2], st[3]
    ptt = (u1 * u1 * st[5] + 2 * u1 * u2 * st[7] + u2 * u2 * st[6]) / (u0 * u0)
    Pn = (ptt - st[5] - st[6]) / ((4 / 3) * st[0])
    Po = pi["ee"] / ((4 / 3) * eo)
    assert np.max(np.abs(Pn[m] - Po[m])) < 1e-3
    assert float(rho_of(tau, 0.0)) > 0  # the centre has passed rho = 0
