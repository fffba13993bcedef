"""The isothermal freeze-out surface (vh_freezeout_2d, host code) on fields
whose isotherm is known: a uniform cooling fluid (the surface is tau =
tau_fo), a static Gaussian (a cylinder r = R_fo), and ideal Gubser flow (the
analytic isotherm and its normal)."""
import ctypes

import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200.hydro import freezeout_2d


def grid(nx, ny, dx, dy):
    gx, gy = nx + 6, ny + 6
    X = -(nx // 2) * dx + (np.arange(gx) - 3) * dx
    Y = -(ny // 2) * dy + (np.arange(gy) - 3) * dy
    YY, XX = np.meshgrid(Y, X, indexing="ij")
    return XX.ravel(), YY.ravel()


def at_rest(n):
    u = np.zeros((3, n))
    u[0] = 1.0
    return u


def test_uniform_cooling_gives_the_plane_tau_fo():
    nx, ny, dx, dy = 20, 16, 0.1, 0.2
    x, _ = grid(nx, ny, dx, dy)
    n = x.size
    t0, t1, tfo = 0.20, 0.14, 0.15
    tau0, tau1 = 2.0, 2.1
    el = freezeout_2d(nx, ny, dx, dy, tau0, tau1, np.full(n, t0), np.full(n, t1), at_rest(n), at_rest(n), tfo)
    tau_fo = tau0 + (t0 - tfo) / (t0 - t1) * (tau1 - tau0)
    assert np.allclose(el[:, 0], tau_fo, rtol=1e-14)
    assert el[:, 3].sum() == pytest.approx(tau_fo * (nx - 1) * (ny - 1) * dx * dy, rel=1e-12)
    assert np.all(el[:, 3] > 0)  # pointing to later times, where it is colder
    assert np.abs(el[:, 4:6]).max() <= 1e-14
    assert np.allclose(el[:, 6], 1.0) and np.abs(el[:, 7:9]).max() == 0


def test_static_gaussian_gives_a_cylinder():
    nx = ny = 81
    dx = dy = 0.1
    x, y = grid(nx, ny, dx, dy)
    T = 0.3 * np.exp(-(x * x + y * y) / (2 * 1.5 ** 2))
    tfo = 0.15
    R = 1.5 * np.sqrt(2 * np.log(0.3 / tfo))
    tau0, tau1 = 1.0, 1.05
    el = freezeout_2d(nx, ny, dx, dy, tau0, tau1, T, T, at_rest(x.size), at_rest(x.size), tfo)
    r = np.hypot(el[:, 1], el[:, 2])
    assert np.abs(r - R).max() <= 5e-3  # the polygon of the linear interpolant
    assert np.abs(el[:, 3]).max() <= 1e-14  # time-like normal absent: the surface does not move
    assert np.all(el[:, 4] * el[:, 1] + el[:, 5] * el[:, 2] > 0)  # outwards, to the cold side
    # tau eps dx dx / 2 summed: tau_mid * (circumference) * (tau1 - tau0)
    area = np.hypot(el[:, 4], el[:, 5]).sum()
    assert area == pytest.approx(0.5 * (tau0 + tau1) * 2 * np.pi * R * (tau1 - tau0), rel=2e-3)


def gubser_T(tau, r, q=1.0, c=1.0):
    return c / (tau ** (1 / 3) * (1 + 2 * q * q * (tau * tau + r * r) + q ** 4 * (tau * tau - r * r) ** 2) ** (1 / 3))


def test_ideal_gubser_isotherm_and_normal():
    nx = ny = 101
    dx = dy = 0.08
    x, y = grid(nx, ny, dx, dy)
    r = np.hypot(x, y)
    tau0, tau1 = 1.2, 1.21
    tfo = 0.5 * gubser_T(1.2, 0.0)
    el = freezeout_2d(nx, ny, dx, dy, tau0, tau1, gubser_T(tau0, r), gubser_T(tau1, r), at_rest(x.size),
                      at_rest(x.size), tfo)
    assert len(el) > 100
    tc, rc = el[:, 0], np.hypot(el[:, 1], el[:, 2])
    assert np.abs(gubser_T(tc, rc) / tfo - 1).max() <= 1e-3
    # the normal against -grad T of the closed form (tau, x, y components)
    h = 1e-6
    gt = (gubser_T(tc + h, rc) - gubser_T(tc - h, rc)) / (2 * h)
    gr = (gubser_T(tc, rc + h) - gubser_T(tc, rc - h)) / (2 * h)
    g = -np.array([gt, gr * el[:, 1] / rc, gr * el[:, 2] / rc]).T
    n = el[:, 3:6]
    cosang = (n * g).sum(axis=1) / (np.linalg.norm(n, axis=1) * np.linalg.norm(g, axis=1))
    assert cosang.min() >= 0.999  # within 2.6 degrees


def test_arguments_and_capacity():
    L = A.lib()
    nx = ny = 8
    n = (nx + 6) * (ny + 6)
    T0, T1, u = np.full(n, 0.2), np.full(n, 0.1), at_rest(n).ravel().copy()
    out = np.zeros((4, 9))
    cnt = ctypes.c_longlong()
    rc = L.vh_freezeout_2d(nx, ny, 0.1, 0.1, 1.0, 1.1, A.ptr(T0), A.ptr(T1), A.ptr(u), A.ptr(u), 0.15, A.ptr(out), 4,
                           ctypes.byref(cnt))
    assert rc == A.E_ARG and cnt.value > 4  # the count is reported although it did not fit
    assert L.vh_freezeout_2d(nx, ny, 0.1, 0.1, 1.1, 1.0, A.ptr(T0), A.ptr(T1), A.ptr(u), A.ptr(u), 0.15, A.ptr(out),
                             4, ctypes.byref(cnt)) == A.E_ARG


def grid3(nx, ny, nz, dx, dy, dz):
    gx, gy, gz = nx + 6, ny + 6, nz + 6
    X = -(nx // 2) * dx + (np.arange(gx) - 3) * dx
    Y = -(ny // 2) * dy + (np.arange(gy) - 3) * dy
    Z = -(nz // 2) * dz + (np.arange(gz) - 3) * dz
    ZZ, YY, XX = np.meshgrid(Z, Y, X, indexing="ij")
    return XX.ravel(), YY.ravel(), ZZ.ravel()


def test_3d_uniform_cooling_gives_the_plane_tau_fo():
    from viral_b200.hydro import freezeout_3d
    nx, ny, nz, dx, dy, dz = 6, 5, 4, 0.1, 0.2, 0.25
    x, _, _ = grid3(nx, ny, nz, dx, dy, dz)
    n = x.size
    u = np.zeros((4, n))
    u[0] = 1.0
    t0, t1, tfo, tau0, tau1 = 0.2, 0.14, 0.15, 2.0, 2.1
    el = freezeout_3d(nx, ny, nz, dx, dy, dz, tau0, tau1, np.full(n, t0), np.full(n, t1), u, u, tfo)
    tau_fo = tau0 + (t0 - tfo) / (t0 - t1) * (tau1 - tau0)
    assert np.allclose(el[:, 0], tau_fo, rtol=1e-14)
    assert el[:, 4].sum() == pytest.approx(tau_fo * (nx - 1) * (ny - 1) * (nz - 1) * dx * dy * dz, rel=1e-12)
    assert np.all(el[:, 4] > 0) and np.abs(el[:, 5:8]).max() <= 1e-14


def test_3d_static_ball_gives_a_sphere():
    """a static Gaussian in (x, y, eta): the surface is a sphere of the
    coordinate space; its dSigma (x, y, eta) point outwards and add up to
    tau 4 pi R^2 (tau1 - tau0)"""
    from viral_b200.hydro import freezeout_3d
    nx = ny = nz = 33
    d = 0.1
    x, y, z = grid3(nx, ny, nz, d, d, d)
    T = 0.3 * np.exp(-(x * x + y * y + z * z) / (2 * 0.6 ** 2))
    tfo = 0.15
    R = 0.6 * np.sqrt(2 * np.log(2.0))
    u = np.zeros((4, x.size))
    u[0] = 1.0
    tau0, tau1 = 1.0, 1.05
    el = freezeout_3d(nx, ny, nz, d, d, d, tau0, tau1, T, T, u, u, tfo)
    r = np.linalg.norm(el[:, 1:4], axis=1)
    assert np.abs(r - R).max() <= 6e-3
    assert np.abs(el[:, 4]).max() <= 1e-14
    assert np.all((el[:, 5:8] * el[:, 1:4]).sum(axis=1) > 0)
    area = np.linalg.norm(el[:, 5:8], axis=1).sum()
    assert area == pytest.approx(0.5 * (tau0 + tau1) * 4 * np.pi * R * R * (tau1 - tau0), rel=1e-2)


def test_cooper_frye_on_known_surfaces():
    """Boltzmann spectra (vh_cooper_frye_2d): a plane tau = tau_fo of a fluid
    at rest gives g A tau_fo 2 m_T K1(m_T/T) / (2 pi)^3 and, integrated, A
    tau_fo times the equilibrium density; a uniformly moving fluid adds its
    Lorentz factor and boost; a static closed cylinder emits nothing net"""
    from scipy import integrate, special
    from viral_b200.hydro import cooper_frye_2d
    nx, ny, dx, dy = 20, 16, 0.1, 0.2
    x, _ = grid(nx, ny, dx, dy)
    n = x.size
    tfo, m, g = 0.15 / 0.19733, 0.14 / 0.19733, 3.0  # fm^-1: 150 MeV, a pion-like mass
    tau0, tau1 = 2.0, 2.1
    el = freezeout_2d(nx, ny, dx, dy, tau0, tau1, np.full(n, 1.2 * tfo), np.full(n, 0.8 * tfo), at_rest(n), at_rest(n),
                      tfo)
    A_tau = el[:, 3].sum()
    pt = np.array([0.5, 1.0, 2.0, 5.0])
    phi = np.linspace(0, 2 * np.pi, 5, endpoint=False)
    sp = cooper_frye_2d(el, tfo, m, g, pt, phi)
    mt = np.sqrt(m * m + pt * pt)
    want = g * A_tau * 2 * mt * special.k1(mt / tfo) / (2 * np.pi) ** 3
    assert np.allclose(sp, want[:, None], rtol=1e-12)
    dndy = integrate.quad(lambda p: 2 * np.pi * p * cooper_frye_2d(el, tfo, m, g, [p], [0.0])[0, 0], 0, 60 * tfo,
                          epsrel=1e-10)[0]
    n_eq = g * m * m * tfo * special.kn(2, m / tfo) / (2 * np.pi ** 2)
    assert dndy == pytest.approx(A_tau * n_eq, rel=1e-7)
    # a uniformly moving fluid: u = (gamma, gamma v, 0)
    v = 0.4
    gam = 1 / np.sqrt(1 - v * v)
    u = np.zeros((3, n))
    u[0], u[1] = gam, gam * v
    el = freezeout_2d(nx, ny, dx, dy, tau0, tau1, np.full(n, 1.2 * tfo), np.full(n, 0.8 * tfo), u, u, tfo)
    sp = cooper_frye_2d(el, tfo, m, g, pt, phi)
    px = pt[:, None] * np.cos(phi)[None, :]
    want = g * A_tau * 2 * mt[:, None] * special.k1(mt[:, None] * gam / tfo) * np.exp(px * gam * v / tfo) / (2 * np.pi) ** 3
    assert np.allclose(sp, want, rtol=1e-12)
    # a static cylinder at rest: the outgoing and incoming halves cancel
    nx = ny = 41
    x, y = grid(nx, ny, 0.1, 0.1)
    T = 0.3 * np.exp(-(x * x + y * y) / (2 * 1.0 ** 2))
    el = freezeout_2d(nx, ny, 0.1, 0.1, 1.0, 1.05, T, T, at_rest(x.size), at_rest(x.size), 0.15)
    sp = cooper_frye_2d(el, 0.15, 0.3, 1.0, [0.2, 0.5], [0.0, 1.0])
    scale = cooper_frye_2d(np.abs(el), 0.15, 0.3, 1.0, [0.2, 0.5], [0.0, 1.0])
    assert np.abs(sp).max() <= 1e-12 * np.abs(scale).max()


def test_cooper_frye_3d_reduces_to_the_boost_invariant_result():
    """a fluid at rest, uniform in x, y, eta over eta in [-6, 6] and cooling
    through T_fo: the 3+1D sum over the surface's eta cells approaches the
    rapidity integral of the boost-invariant formula (2 m_T K1) at y = 0
    (the midpoint rule in eta converges geometrically for this integrand)"""
    from scipy import special
    from viral_b200.hydro import cooper_frye_3d, freezeout_3d
    nx, ny, nz, dx, dy, dz = 4, 4, 121, 0.2, 0.2, 0.1
    x, _, _ = grid3(nx, ny, nz, dx, dy, dz)
    n = x.size
    u = np.zeros((4, n))
    u[0] = 1.0
    tfo, m, g = 0.76, 0.71, 1.0
    el = freezeout_3d(nx, ny, nz, dx, dy, dz, 2.0, 2.1, np.full(n, 1.1 * tfo), np.full(n, 0.9 * tfo), u, u, tfo)
    A_tau = el[:, 4].sum() / ((nz - 1) * dz)  # per unit rapidity
    pt = np.array([0.3, 1.0, 3.0])
    sp = cooper_frye_3d(el, tfo, m, g, 0.0, pt, [0.0, 1.0])
    mt = np.sqrt(m * m + pt * pt)
    want = g * A_tau * 2 * mt * special.k1(mt / tfo) / (2 * np.pi) ** 3
    assert np.allclose(sp, want[:, None], rtol=1e-10)


def test_flow_coefficients_of_spectra():
    """v_n and the event-plane angles of a spectrum with known harmonics, and
    the elliptic flow of an elliptic fireball's spectrum: positive, rising
    with p_T, its plane along the short axis (x)"""
    from viral_b200.hydro import cooper_frye_2d, flow_coefficients
    phi = np.arange(16) * 2 * np.pi / 16
    pt = np.array([0.5, 1.0])
    amp = np.array([[1.0], [0.3]])
    S = amp * (1 + 2 * 0.1 * np.cos(2 * (phi - 0.3)) + 2 * 0.05 * np.cos(3 * (phi + 0.2)))[None, :]
    v, psi = flow_coefficients(S, phi, orders=(1, 2, 3))
    assert np.allclose(v[0], 0, atol=1e-15) and np.allclose(v[1], 0.1) and np.allclose(v[2], 0.05)
    assert np.allclose(psi[1], 0.3) and np.allclose(psi[2], -0.2)
    with pytest.raises(ValueError):
        flow_coefficients(S, phi[:-1])

    # an elliptic fireball expanding faster along x (its short axis)
    nx = ny = 61
    d = 0.1
    x, y = grid(nx, ny, d, d)
    T = 0.3 * np.exp(-(x * x / 1.0 + y * y / 2.0) / 2)
    u = np.stack([np.sqrt(1 + (0.6 * x) ** 2 + (0.3 * y) ** 2), 0.6 * x, 0.3 * y])
    el = freezeout_2d(nx, ny, d, d, 1.0, 1.05, T, 0.97 * T, u, u, 0.15)
    pts = np.array([0.5, 1.0, 2.0])
    v, psi = flow_coefficients(cooper_frye_2d(el, 0.15, 0.14, 1.0, pts, phi), phi, orders=(2,))
    assert np.all(v[0] > 0) and np.all(np.diff(v[0]) > 0)
    # the tetrahedra's diagonal breaks the x -> -x mirror symmetry slightly
    assert np.allclose(psi[0], 0.0, atol=2e-3)
