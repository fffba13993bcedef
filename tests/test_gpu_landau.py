"""Landau matching on the GPU (vh_landau_match) and the initial state from
T^{mu nu} (vh_init_tmunu) through the C ABI."""
import numpy as np
import pytest

from test_landau_cpu import IDX, find_var, fluid_tensor
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Hydro, landau_match

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cart", [False, True])
def test_landau_match_recovers_fluid_tensors(cart):
    rng = np.random.default_rng(8)
    tau = 1.0 if cart else 1.7
    cols, es, us = [], [], []
    for _ in range(3000):
        T10, e, u = fluid_tensor(rng, tau, cart, rng.uniform(0.2, 100))
        cols.append(T10); es.append(e); us.append(u)
    T = np.array(cols).T.copy()
    e, u, nfail = landau_match(T, tau, cart)
    assert nfail == 0
    assert np.max(np.abs(e - np.array(es)) / np.array(es)) <= 1e-12
    U = np.array(us).T
    assert np.max(np.abs(u - U) / U[0]) <= 1e-11
    for c in range(0, 3000, 300):
        (E, v), = find_var(T[:, c], tau, cart, scaled=True)
        assert abs(E - e[c]) <= 1e-12 * E


def test_landau_match_reports_failures():
    T = np.array([[1.0, 20.0], [2.0, 1.0], [0, 0], [0, 0], [1.0, 7.0], [0, 0], [0, 0], [0.3, 7.0], [0, 0],
                  [0.3, 6.0]])
    e, u, nfail = landau_match(T, 1.0, True)
    assert nfail == 1
    (E, v), = find_var(T[:, 1], 1.0, True)
    assert abs(e[1] - E) <= 1e-12 * E and np.max(np.abs(u[1:, 1] / u[0, 1] - v)) <= 1e-12


def tmunu_of(p, tau, cart=False):
    """the fluid tensor of (e, P, u, pi), with u^tau the normalisation of the
    spatial u (the Gubser test's mirrored ghost cells store another u^tau)"""
    t2 = 1.0 if cart else tau * tau
    gi = [1.0, -1.0, -1.0, -1.0 / t2]
    u = p["u"].copy()
    u[0] = np.sqrt(1 + u[1] ** 2 + u[2] ** 2 + t2 * u[3] ** 2)
    out = np.zeros((10, u.shape[1]))
    for q, (a, b) in enumerate(IDX):
        out[q] = (p["e"] + p["P"]) * u[a] * u[b] + p["pi"][q] - (p["P"] * gi[a] if a == b else 0.0)
    return out


@pytest.mark.parametrize("which", ["gubser", "glauber3d"])
def test_init_tmunu_round_trip(which):
    """T^{mu nu} of an evolved viscous state, matched back: e and u of the
    state; pi and T^{tau mu} of the state for the conformal EOS (Gubser),
    and with the reference's trace correction otherwise: its pi is
    T - T_id - PI (g - u u) with PI = -(e - 3P)/3, which adds (e - 3P)/3
    (g - u u) to a fluid tensor's pi (NEWEST5/ginit.h:955-989)"""
    if which == "gubser":
        cfg = C.gubser_config(nx=33, ny=33)
        inp = C.gubser_inputs(cfg)
    else:
        cfg = C.glauber_config(nx=20, ny=18, nz=10, boost_invariant=False)
        inp = C.glauber_inputs(cfg, b=5.0, seed=2)
    with C.make_hydro(cfg, inp) as H:
        H.step(6)
        tau = H.tau
        s = H.get_state()
        p = H.get_primitive()
    # ghost cells get the ideal-fluid tensor of their (e, u): the Gubser
    # test's corner ghosts keep a pi that no fluid tensor has
    from helpers import interior_mask
    p["pi"][:, ~interior_mask(cfg)] = 0.0
    T = tmunu_of(p, tau)
    with Hydro(cfg) as H2:
        assert H2.init_tmunu(tau, T) == 0
        s2 = H2.get_state()
        assert abs(H2.tau - tau) < 1e-15
    if which != "gubser":
        # the expected state: pi + (e - 3P)/3 (g - u u), T^{tau mu} by the
        # oracle's closure of it
        from helpers import oracle_config
        from pyoracle import Oracle
        t2 = tau * tau
        gi = [1.0, -1.0, -1.0, -1.0 / t2]
        u = s[1:5]
        tr = (s[0] - 3 * p["P"]) / 3
        for m, (a, b) in enumerate([(1, 1), (2, 2), (1, 2), (1, 3), (2, 3)]):
            s[5 + m] = s[5 + m] + tr * ((gi[a] if a == b else 0.0) - u[a] * u[b])
        O = Oracle(oracle_config(cfg))
        O.set_state(s)
        O.fill_tmunu(tau)
        s = O.get_state()
    # interior cells (the Gubser test's mirrored ghosts hold a u^tau that is
    # not the normalisation of their u^x, u^y)
    m = interior_mask(cfg)
    for grp in ((0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13)):
        scale = max(np.max(np.abs(s[q][m])) for q in grp)
        for q in grp:
            assert np.max(np.abs(s2[q][m] - s[q][m])) <= 1e-11 * scale, q
    assert np.array_equal(s2[14:18], s2[1:5])  # prevu = u
