"""Named workloads of the viscous KT step and their inputs.

gubser_129        boost-invariant Gubser test: 129x129, dx = 0.1 fm, q = 1/fm,
                  tau0 = 1 fm/c, T(0,0) = 0.6 GeV, conformal e = a T^4,
                  eta/s = 0.2, tau_pi = 5 eta/(e+P), Navier-Stokes pi,
                  dtau = 0.01 fm/c to tau = 4 fm/c (300 steps), mirrored
                  u^x,u^y ghosts as the reference's Gubser scenario.
glauber_161x161x41 3+1D Milne event: 161x161x41, dx = dy = 0.1 fm,
                  d eta = 0.25, tau0 = 0.6 -> 10 fm/c, dtau = 0.02 (470 steps),
                  MC-Glauber Pb+Pb b = 7 fm (seed 0), synthetic EOS table,
                  eta/s = 0.08, tau_pi = 1.5 eta/P, u = 0, pi = 0.
bjorken           the reference's Bjorken block: a uniform fluid at rest in
                  Milne coordinates, 10x10 cells, e = 30 GeV/fm^3 at 0.6 fm/c,
                  eta = 0.2 s, tau_pi = 0.01 fm/c (bjorken_config/_inputs).
cart_bjorken      the reference's Cartesian Bjorken block: the same fluid at
                  rest in (t, x, y, z), 10x10x41 cells of 0.1 fm from
                  t = 0.6 (cart_bjorken_config/_inputs), an equilibrium.
The reference's cold-plasma Gubser test and its Glasma initial state come
from the generators in hydro.py (profile_gubser_cold, profile_cgc).
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi as A
from .hydro import A_QGP, HBARC, Config, eos_table_synthetic, profile_glauber, profile_gubser

_EOS_CACHE: dict = {}


def eos_table() -> np.ndarray:
    if "t" not in _EOS_CACHE:
        _EOS_CACHE["t"] = eos_table_synthetic(2000, 1e-3, 500.0, A_QGP, HBARC)
    return _EOS_CACHE["t"]


BJORKEN_GEVFM = 0.1973                     # the reference's GEVFM (NEWEST5/main.cpp:46)
BJORKEN_A = 3 * 42.25 * math.pi ** 2 / 90  # FACTOR, DOF = 42.25 (NEWEST5/maindef.h)
BJORKEN_E0 = 30.0 / BJORKEN_GEVFM           # 30 GeV/fm^3 (NEWEST5/init.h:292)


def bjorken_config(nx=10, ny=10, precision=A.PREC_FP64) -> Config:
    """The reference's Bjorken scenario block (NEWEST5/maindef.h:195-235):
    a uniform boost-invariant fluid, 10x10 cells of 0.1 fm, tau0 = 0.6 fm/c,
    dtau = 0.01, conformal e = a T^4 with 42.25 degrees of freedom,
    eta = 0.2 s, tau_pi = 0.01 fm/c."""
    return Config(nx=nx, ny=ny, nz=1, boost_invariant=True, precision=precision, dx=0.1, dy=0.1, tau0=0.6,
                  dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=BJORKEN_A, etas0=0.2, etas1=0.0,
                  hbarc=BJORKEN_GEVFM, taupi_kind=A.TAUPI_CONST, taupi_const=0.01)


def cart_bjorken_config(precision=A.PREC_FP64) -> Config:
    """The reference's Cartesian Bjorken block (TXYZ5/maindef.h:78-108): 10x10x41
    cells of 0.1 fm, t0 = 0.6, dt = 0.01, the Milne block's EOS and transport."""
    return Config(nx=10, ny=10, nz=41, boost_invariant=False, coords=A.COORD_CARTESIAN, precision=precision, dx=0.1,
                  dy=0.1, dz=0.1, tau0=0.6, dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=BJORKEN_A, etas0=0.2,
                  etas1=0.0, hbarc=BJORKEN_GEVFM, taupi_kind=A.TAUPI_CONST, taupi_const=0.01)


def cart_bjorken_inputs(cfg: Config):
    """TXYZ5/init.h:221-283: e = 30 GeV/fm^3 at rest on every cell, prevu = u,
    pi = 0"""
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz
    z = np.zeros(n)
    return dict(tau=cfg.tau0, e=np.full(n, BJORKEN_E0), ux=z, uy=z.copy(), ueta=z.copy(), prevu=None,
                pi_mode=A.PI_ZERO)


def bjorken_inputs(cfg: Config):
    """NEWEST5/init.h:283-340: e = 30 GeV/fm^3 on every cell, at rest in
    Milne coordinates (Bjorken flow), prevu = u, pi = 0."""
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz
    z = np.zeros(n)
    return dict(tau=cfg.tau0, e=np.full(n, BJORKEN_E0), ux=z, uy=z.copy(), ueta=None, prevu=None, pi_mode=A.PI_ZERO)


def gubser_config(nx=129, ny=129, dx=0.1, precision=A.PREC_FP64, recon=A.RECON_WENO5) -> Config:
    return Config(nx=nx, ny=ny, nz=1, boost_invariant=True, precision=precision, recon=recon, dx=dx, dy=dx,
                  tau0=1.0, dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=A_QGP, etas0=0.2, etas1=0.0,
                  taupi_kind=A.TAUPI_5_ETA_OVER_EPP, gubser_mirror=True)


def gubser_inputs(cfg: Config, t0_gev=0.6, q=1.0):
    e, ux, uy, pu = profile_gubser(cfg.nx, cfg.ny, cfg.dx, cfg.dy, q, cfg.tau0, cfg.dtau, t0_gev, cfg.eos_a,
                                   cfg.hbarc)
    return dict(tau=cfg.tau0, e=e, ux=ux, uy=uy, ueta=None, prevu=pu, pi_mode=A.PI_NS)


def glauber_config(nx=161, ny=161, nz=41, boost_invariant=False, precision=A.PREC_FP64, dx=0.1, deta=0.25,
                   tau0=0.6, dtau=0.02, etas0=0.08, etas1=0.0, recon=A.RECON_WENO5) -> Config:
    return Config(nx=nx, ny=ny, nz=(1 if boost_invariant else nz), boost_invariant=boost_invariant,
                  precision=precision, recon=recon, dx=dx, dy=dx, dz=deta, tau0=tau0, dtau=dtau,
                  eos_kind=A.EOS_TABLE, eos_table=eos_table(), etas0=etas0, etas1=etas1, etas_tc=0.154,
                  taupi_kind=A.TAUPI_15_ETA_OVER_P)


# Initial energy-density floor (GeV/fm^3), 5e-3 of the 40 GeV/fm^3 peak.
# The near-vacuum outside the fireball has no regulator in the reference, and
# whether the 161x161x41 event reaches tau = 10 fm/c without a failed
# root-find there depends on the floor, not monotonically (measured: 0.04
# fails in one mixed-precision build at tau = 7.48, 0.1 fails in FP64 and
# mixed at tau = 9.8; 0.08 and 0.2 run through in both).
GLAUBER_FLOOR_GEV = 0.2
# Floor of the batched-ensemble events (boost-invariant, to tau = 15 fm/c).
# Of 2048 events, 268 end in a failed root-find (|v| -> 1 at the box edge)
# with 0.04 GeV/fm^3, 82 with 0.1, 50 with 0.5 (mixed; FP64: 55).
ENSEMBLE_FLOOR_GEV = 0.5


def glauber_inputs(cfg: Config, b=7.0, seed=0, efloor_gev=None):
    floor = GLAUBER_FLOOR_GEV if efloor_gev is None else efloor_gev
    e, npart = profile_glauber(cfg.nx, cfg.ny, cfg.nz, cfg.boost_invariant, cfg.dx, cfg.dy, cfg.dz, b=b, seed=seed,
                               efloor_gev=floor, hbarc=cfg.hbarc)
    z = np.zeros_like(e)
    return dict(tau=cfg.tau0, e=e, ux=z, uy=z, ueta=z, prevu=None, pi_mode=A.PI_ZERO, npart=npart)


# The adjoint workload: boost-invariant 128x128 event, b = 7 fm, seed 0,
# eta/s(T) = 0.08 + 1.0 GeV^-1 max(T - 0.154 GeV, 0), 330 steps from 0.6 to
# 7.2 fm/c.  Its floor is 0.5 GeV/fm^3: with 0.04 the near-vacuum edge makes
# eps_p non-smooth at the 1e-6 scale (central differences with h = 1e-6 miss
# the derivative by O(1) and reach it only at h <= 1e-9).
ADJOINT_FLOOR_GEV = 0.5
ADJOINT_STEPS = 330


def adjoint_config(side=128, precision=A.PREC_FP64, c0=0.08, c1=1.0) -> Config:
    return glauber_config(nx=side, ny=side, boost_invariant=True, precision=precision, etas0=c0, etas1=c1)


def adjoint_inputs(cfg: Config, b=7.0, seed=0):
    return glauber_inputs(cfg, b=b, seed=seed, efloor_gev=ADJOINT_FLOOR_GEV)


def make_hydro(cfg: Config, inputs: dict):
    from .hydro import Hydro
    h = Hydro(cfg)
    h.init_profile(inputs["tau"], inputs["e"], inputs["ux"], inputs["uy"], inputs.get("ueta"), inputs.get("prevu"),
                   inputs["pi_mode"], inputs.get("pi5"))
    return h


def steps_between(t0: float, t1: float, dt: float) -> int:
    return int(math.floor((t1 - t0) / dt + 0.5))
