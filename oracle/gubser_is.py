"""Semi-analytic Israel-Stewart Gubser flow: the known answer of the
reference's viscous Gubser test (NEWEST5/init.h:413-550 reads its initial
state from a table, init/tempbin-23F.dat, which the reference does not ship;
its init/tempbin-8.7z is an archive of another such table).  TEST
INFRASTRUCTURE ONLY: the checker of the GPU runs, never on the product path.

Conformal fluid, e = a T^4, constant eta/s, tau_pi = 5 eta/(e+P)
(NEWEST5/maindef.h:338-339), Gubser flow with parameter q.  In the de
Sitter time rho, sinh rho = -(1 - q^2 tau^2 + q^2 r^2)/(2 q tau), the fluid
is at rest and T^ = tau T and P = tau^2 pi^{eta eta}/(e + P_pressure)
depend on rho alone:
    d ln T^/d rho = -(2/3) tanh rho + (1/3) P tanh rho
    dP/d rho      = -(4/3) P^2 tanh rho - P T^/(5 eta/s) + (4/15) tanh rho
(energy conservation with theta^ = 2 tanh rho and pi^{mu nu} sigma_{mu nu}
= pi^{eta eta} tanh rho; the relaxation equation tau_pi (D pi + (4/3) pi
theta) + pi = 2 eta sigma with sigma^{eta eta} = (2/3) tanh rho in the
reference's mostly-minus convention).  Integrated here with SciPy's DOP853
at rtol 1e-12 (the product's generator uses its own RK4).  The reference's
shipped table is this solution with T^ = 1.2, P = 0 at rho = 0 and
eta/s = 0.2 (tests/test_gubser_is_cpu.py checks it to the table's digits).

In Milne coordinates the rest-frame shear is w P along eta (orthonormal) and
-w P/2 along phi and along n = (sinh k, cosh k cos phi, cosh k sin phi), the
unit vector of the (tau, r) plane orthogonal to u = (cosh k, sinh k cos phi,
sinh k sin phi), tanh k = 2 q^2 tau r/(1 + q^2 tau^2 + q^2 r^2).
"""
from __future__ import annotations

import math

import numpy as np


def rho_of(tau, r, q=1.0):
    return np.arcsinh(-(1 - q * q * tau * tau + q * q * r * r) / (2 * q * tau))


class GubserIS:
    """T^(rho) and P(rho) through (rho0, T^0, P0)."""

    def __init__(self, t_hat0: float, p0: float = 0.0, etas: float = 0.2, rho0: float = 0.0,
                 rho_range=(-6.0, 4.0)):
        from scipy.integrate import solve_ivp
        self.etas = etas

        def f(x, y):
            th = math.tanh(x)
            return [-(2 / 3) * th + (1 / 3) * y[1] * th,
                    -(4 / 3) * y[1] * y[1] * th - y[1] * math.exp(y[0]) / (5 * etas) + (4 / 15) * th]

        y0 = [math.log(t_hat0), p0]
        kw = dict(method="DOP853", rtol=1e-12, atol=1e-14, dense_output=True)
        self.dn = solve_ivp(f, [rho0, rho_range[0]], y0, **kw) if rho_range[0] < rho0 else None
        self.up = solve_ivp(f, [rho0, rho_range[1]], y0, **kw) if rho_range[1] > rho0 else None
        self.rho0 = rho0

    def __call__(self, rho):
        rho = np.asarray(rho, dtype=float)
        lt = np.empty_like(rho)
        p = np.empty_like(rho)
        lo = rho < self.rho0
        if np.any(lo):
            y = self.dn.sol(rho[lo])
            lt[lo], p[lo] = y[0], y[1]
        if np.any(~lo):
            y = self.up.sol(rho[~lo])
            lt[~lo], p[~lo] = y[0], y[1]
        return np.exp(lt), p


def milne_fields(sol: GubserIS, tau, x, y, a, q=1.0):
    """T (fm^-1), e, u^mu (4) and pi^{mu nu} (dict of tt, tx, ty, xx, xy, yy,
    ee = tau^2 pi^{eta eta}) at time tau on points x, y"""
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    r = np.sqrt(x * x + y * y)
    th, p = sol(rho_of(tau, r, q))
    T = th / tau
    e = a * T ** 4
    w = (4 / 3) * e
    k = np.arctanh(2 * q * q * tau * r / (1 + q * q * tau * tau + q * q * r * r))
    ch, sh = np.cosh(k), np.sinh(k)
    with np.errstate(invalid="ignore", divide="ignore"):
        cphi = np.where(r > 0, x / np.where(r > 0, r, 1), 1.0)
        sphi = np.where(r > 0, y / np.where(r > 0, r, 1), 0.0)
    n = np.stack([sh, ch * cphi, ch * sphi])       # tau, x, y components of n
    f = np.stack([np.zeros_like(r), -sphi, cphi])  # of e_phi
    hp = -0.5 * w * p
    pi = {}
    names = {"tt": (0, 0), "tx": (0, 1), "ty": (0, 2), "xx": (1, 1), "xy": (1, 2), "yy": (2, 2)}
    for nm, (a_, b_) in names.items():
        pi[nm] = hp * (n[a_] * n[b_] + f[a_] * f[b_])
    pi["ee"] = w * p
    u = np.stack([ch, sh * cphi, sh * sphi, np.zeros_like(r)])
    return T, e, u, pi
