"""Shared helpers of the test suite: the oracle configuration matching a
product Config, canonical states from profile inputs, interior masks."""
from __future__ import annotations

import numpy as np

from pyoracle import Oracle, OracleConfig, grid_coords, smooth_state  # noqa: F401
from viral_b200 import _abi as A
from viral_b200.hydro import Config


def oracle_config(cfg: Config) -> OracleConfig:
    return OracleConfig(nx=cfg.nx, ny=cfg.ny, nz=(1 if cfg.boost_invariant else cfg.nz),
                        boost_invariant=cfg.boost_invariant, cartesian=cfg.coords == A.COORD_CARTESIAN,
                        dx=cfg.dx, dy=cfg.dy, dz=cfg.dz, eos_kind=cfg.eos_kind, eos_a=cfg.eos_a,
                        eos_table=cfg.eos_table, etas0=cfg.etas0, etas1=cfg.etas1, etas_tc=cfg.etas_tc,
                        hbarc=cfg.hbarc, taupi_kind=cfg.taupi_kind, gubser_mirror=cfg.gubser_mirror,
                        recon=cfg.recon, minmod_theta=cfg.minmod_theta, taupi_const=cfg.taupi_const,
                        cold_plasma=cfg.cold_plasma)


def canonical_state(cfg: Config, inp: dict) -> np.ndarray:
    """18-field state from profile inputs with pi = 0 and T^{tau mu} unset
    (the oracle's fill_tmunu / ns_init completes it)."""
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz
    tau = inp["tau"]
    t2 = 1.0 if cfg.coords == A.COORD_CARTESIAN else tau * tau
    f = np.zeros((18, n))
    ue = inp.get("ueta")
    ue = np.zeros(n) if ue is None else np.asarray(ue).reshape(n)
    f[0] = np.asarray(inp["e"]).reshape(n)
    f[2] = np.asarray(inp["ux"]).reshape(n)
    f[3] = np.asarray(inp["uy"]).reshape(n)
    f[4] = ue
    f[1] = np.sqrt(1 + f[2] ** 2 + f[3] ** 2 + t2 * f[4] ** 2)
    pu = inp.get("prevu")
    f[14:18] = f[1:5] if pu is None else np.asarray(pu).reshape(4, n)
    return f


def oracle_from_inputs(cfg: Config, inp: dict) -> Oracle:
    O = Oracle(oracle_config(cfg))
    O.set_state(canonical_state(cfg, inp))
    if inp["pi_mode"] == A.PI_NS:
        O.ns_init(inp["tau"], cfg.dtau)
    else:
        O.fill_tmunu(inp["tau"])
    return O


def interior_mask(cfg: Config) -> np.ndarray:
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz
    idx = np.arange(n)
    i = idx % gx
    j = (idx // gx) % gy
    k = idx // (gx * gy)
    kl, kr = (0, 1) if cfg.boost_invariant else (3, 3 + cfg.nz)
    return (i >= 3) & (i < 3 + cfg.nx) & (j >= 3) & (j < 3 + cfg.ny) & (k >= kl) & (k < kr)


def smooth_inputs(cfg: Config, tau: float, seed: int, amp: float = 1.0) -> np.ndarray:
    """A seeded smooth viscous state with T^{tau mu} filled by the oracle."""
    gx, gy, gz = cfg.gdims()
    x, y, z = grid_coords(gx, gy, gz, cfg.dx, cfg.dy, cfg.dz, cfg.boost_invariant)
    cart = cfg.coords == A.COORD_CARTESIAN
    f = smooth_state(x, y, z, tau, cfg.dtau, seed=seed, amp=amp, cartesian=cart)
    O = Oracle(oracle_config(cfg))
    O.set_state(f)
    O.fill_tmunu(tau)
    return O.get_state()


def shock_tube_fixture():
    """The Cartesian shock tube of the reference's default TXYZ5 block
    (TXYZ5/init.h:151-210: e = 16 fm^-4 for z < 0, 1 fm^-4 for z >= 0, at
    rest, pi = 0) and the reference's state after 20 steps, as stored in
    tests/golden/ref_cart_3d_shock.npz.  Returns (fixture, OracleConfig,
    initial 18-field state)."""
    import math
    import os

    from pyoracle import Oracle, OracleConfig, grid_coords
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cart_3d_shock.npz"))
    gx, gy, gz, bi = (int(v) for v in g["dims"])
    dx, dy, dz, factor, gevfm = (float(v) for v in g["consts"])
    cfg = OracleConfig(nx=gx - 6, ny=gy - 6, nz=gz - 6, boost_invariant=False, cartesian=True, dx=dx, dy=dy, dz=dz,
                       eos_kind=0, eos_a=factor, etas0=0.01 / (4 * math.pi), hbarc=gevfm, taupi_kind=0)
    x, y, z = grid_coords(gx, gy, gz, dx, dy, dz, False)
    f = np.zeros((18, gx * gy * gz))
    f[0] = np.where(z < 0, 16.0, 1.0)
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(0.0)
    return g, cfg, O.get_state()
