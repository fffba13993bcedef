"""The reference's analytic viscous known answer: the cold-plasma Gubser flow
(COLDPLASMA, NEWEST5/init.h:489-512 with the shear source of
NEWEST5/Source.h:371-410, which drops the relaxation -pi/tau_pi).  The
oracle, pinned to the compiled reference's cold-plasma source by
tests/golden/ref_gubser_cold.npz, evolves vh_profile_gubser_cold's initial
state and follows the closed form
T = T^(rho)/tau, T^ = 1.21 sech(rho)^(2/3) cosh(4 ln cosh rho / (3 sqrt 5))^(1/4),
sinh rho = -(1 - tau^2 + r^2)/(2 tau), to the discretisation error; the same
run with the ordinary source misses it by five times more."""
import numpy as np
import pytest

from helpers import canonical_state, oracle_config
from pyoracle import Oracle
from viral_b200 import _abi as A
from viral_b200.hydro import Config, profile_gubser_cold

A_CONF = 3 * 42.25 * np.pi ** 2 / 90
K = 4 / (3 * np.sqrt(5))


def closed_form_T(r, tau):
    rho = np.arcsinh(-(1 - tau * tau + r * r) / (2 * tau))
    lc = np.log(np.cosh(rho))
    return 1.21 * np.cosh(K * lc) ** 0.25 / np.cosh(rho) ** (2 / 3) / tau


def cold_config(nx, dx, dt, cold=True):
    return Config(nx=nx, ny=nx, nz=1, boost_invariant=True, dx=dx, dy=dx, tau0=1.0, dtau=dt,
                  eos_kind=A.EOS_CONFORMAL, eos_a=A_CONF, etas0=0.2, etas1=0.0, taupi_kind=A.TAUPI_5_ETA_OVER_EPP,
                  gubser_mirror=True, cold_plasma=cold, hbarc=0.1973)


def initial_state(cfg):
    e, ux, uy, pi5, pu = profile_gubser_cold(cfg.nx, cfg.ny, cfg.dx, cfg.dy, 1.0, cfg.tau0, cfg.dtau, 1.21, A_CONF)
    f = canonical_state(cfg, dict(tau=cfg.tau0, e=e, ux=ux, uy=uy, prevu=pu))
    f[5:10] = pi5
    return f


def radius(cfg):
    gx = cfg.nx + 6
    X = -(cfg.nx // 2) * cfg.dx + (np.arange(gx) - 3) * cfg.dx
    XX, YY = np.meshgrid(X, X)
    return np.hypot(XX, YY).ravel()


def run_oracle(cfg, steps):
    O = Oracle(oracle_config(cfg))
    O.set_state(initial_state(cfg))
    O.fill_tmunu(cfg.tau0)
    tau = cfg.tau0
    for _ in range(steps):
        assert O.step(tau, cfg.dtau) == 0
        tau += cfg.dtau
    return O.get_state(), tau


def test_initial_state_is_the_closed_form():
    cfg = cold_config(41, 0.1, 0.01)
    f = initial_state(cfg)
    r = radius(cfg)
    assert np.max(np.abs((f[0] / A_CONF) ** 0.25 / closed_form_T(r, 1.0) - 1)) <= 1e-14
    # the x-y block of pi has its principal axes along r and phi (u is radial)
    ux, uy = f[2], f[3]
    assert np.max(np.abs(f[7] * (ux ** 2 - uy ** 2) - (f[5] - f[6]) * ux * uy)) <= 1e-12 * np.max(np.abs(f[5]))


def test_oracle_follows_the_closed_form():
    cfg = cold_config(61, 0.1, 0.01)
    s, tau = run_oracle(cfg, 20)
    r = radius(cfg)
    m = r < 1.5
    err = np.max(np.abs((s[0][m] / A_CONF) ** 0.25 / closed_form_T(r[m], tau) - 1))
    ordinary, _ = run_oracle(cold_config(61, 0.1, 0.01, cold=False), 20)
    err_ord = np.max(np.abs((ordinary[0][m] / A_CONF) ** 0.25 / closed_form_T(r[m], tau) - 1))
    print("cold plasma to tau = 1.2: T within %.2e of the closed form (ordinary source %.2e)" % (err, err_ord))
    assert err <= 5e-4 and err_ord >= 3 * err
