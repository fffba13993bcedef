"""Landau matching (the reference's FindVar, NEWEST5/ginit.h:521-656) on the
CPU: the __host__ __device__ function the GPU kernels run, through
libvh_check.so, against a restatement of the reference's selection of the
eigenpair (all four eigenpairs of T^mu_nu, the one real pair whose
eigenvector has |v| < 1)."""
import ctypes

import numpy as np
import pytest

from viral_b200 import build

_dp = ctypes.POINTER(ctypes.c_double)
IDX = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]


@pytest.fixture(scope="module")
def L():
    lib = ctypes.CDLL(build.build_check())
    lib.vhc_landau.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp, _dp]
    lib.vhc_landau.restype = ctypes.c_int
    return lib


def find_var(T10, tau, cart, scaled=False):
    """the reference's FindVar: eigenpairs of T^mu_nu, the real ones with a
    real eigenvector, vec[0] != 0 and |v| < 1; E = |lambda|.  The reference
    tests v^eta = u^eta/u^tau as it is; scaled=True tests the physical
    tau u^eta/u^tau instead (the timelike condition in the Milne metric)."""
    t2 = 1.0 if cart else tau * tau
    g = np.array([1.0, -1.0, -1.0, -t2])
    T = np.zeros((4, 4))
    for q, (a, b) in enumerate(IDX):
        T[a, b] = T[b, a] = T10[q]
    M = T * g[None, :]
    w, V = np.linalg.eig(M)
    found = []
    for i in range(4):
        if np.imag(w[i]) != 0 or np.any(np.imag(V[:, i]) != 0) or np.real(V[0, i]) == 0:
            continue
        v = np.real(V[1:, i]) / np.real(V[0, i])
        vt = v * np.array([1.0, 1.0, np.sqrt(t2)]) if scaled else v
        if np.all(np.abs(vt) < 1) and np.sqrt(np.sum(vt * vt)) < 1:
            found.append((abs(np.real(w[i])), v))
    return found


def fluid_tensor(rng, tau, cart, e, vmax=0.8, pi_frac=0.3):
    """T^{mu nu} = (e + P) u u - P g^{mu nu} + pi with a transverse traceless pi"""
    t2 = 1.0 if cart else tau * tau
    gi = np.diag([1.0, -1.0, -1.0, -1.0 / t2])
    g = np.diag([1.0, -1.0, -1.0, -t2])
    v = rng.uniform(-1, 1, 3)
    v *= vmax * rng.uniform(0, 1) / np.linalg.norm(v)
    # u^eta from the physical velocity tau v^eta
    ui = np.array([v[0], v[1], v[2] / np.sqrt(t2)])
    gam = 1 / np.sqrt(1 - np.sum(v * v))
    u = gam * np.array([1.0, *ui])
    P = e / 3
    D = gi - np.outer(u, u)                      # Delta^{mu nu}
    Dm = D @ g                                   # Delta^mu_nu
    X = rng.normal(size=(4, 4)); X = X + X.T
    pi = Dm @ X @ Dm.T                           # transverse
    tr = np.einsum("ab,ab", g, pi)
    pi = pi - tr / 3 * D                         # traceless
    pi *= pi_frac * P / np.max(np.abs(pi))
    T = (e + P) * np.outer(u, u) - P * gi + pi
    return np.array([T[a, b] for a, b in IDX]), e, u


@pytest.mark.parametrize("cart", [False, True])
def test_fluid_tensors(L, cart):
    rng = np.random.default_rng(3 if cart else 4)
    for trial in range(200):
        tau = 1.0 if cart else rng.uniform(0.3, 3.0)
        T10, e, u = fluid_tensor(rng, tau, cart, rng.uniform(0.5, 80))
        ee = ctypes.c_double(); uu = np.zeros(4)
        ok = L.vhc_landau(T10.ctypes.data_as(_dp), tau, int(cart), ctypes.byref(ee), uu.ctypes.data_as(_dp))
        assert ok == 1
        assert abs(ee.value - e) <= 1e-12 * e
        assert np.max(np.abs(uu - u)) <= 1e-11 * u[0]
        (E, v), = find_var(T10, tau, cart, scaled=True)
        assert abs(ee.value - E) <= 1e-12 * E
        assert np.max(np.abs(uu[1:] / uu[0] - v)) <= 1e-11
        ref = find_var(T10, tau, cart)
        # the reference tests |u^eta/u^tau| < 1 without the factor tau: away
        # from tau = 1 it can keep a spacelike pair as well, or drop the
        # timelike one, and then stops; where it finds one pair, it is ours
        if len(ref) == 1:
            assert abs(ref[0][0] - E) <= 1e-12 * E
        else:
            assert not cart and tau != 1.0


def test_anisotropic_tensor(L):
    """a pressure-anisotropic tensor at rest, then boosted: P_L = 0, P_T = e/2"""
    e = 20.0
    Tr = np.diag([e, e / 2, e / 2, 0.0])
    for vx in (0.0, 0.3, 0.7):
        gam = 1 / np.sqrt(1 - vx * vx)
        B = np.eye(4); B[0, 0] = B[1, 1] = gam; B[0, 1] = B[1, 0] = gam * vx
        T = B @ Tr @ B.T
        T10 = np.array([T[a, b] for a, b in IDX])
        ee = ctypes.c_double(); uu = np.zeros(4)
        assert L.vhc_landau(T10.ctypes.data_as(_dp), 1.0, 1, ctypes.byref(ee), uu.ctypes.data_as(_dp)) == 1
        assert abs(ee.value - e) <= 1e-12 * e and abs(uu[1] / uu[0] - vx) <= 1e-12
        (E, v), = find_var(T10, 1.0, True)
        assert abs(E - ee.value) <= 1e-12 * e


def test_no_timelike_eigenvector(L):
    """energy flux above the energy density: no timelike eigenpair (the
    reference prints EIGEN VALUE SEARCH FAILED and exits)"""
    T10 = np.array([1.0, 2.0, 0, 0, 1.0, 0, 0, 0.3, 0, 0.3])
    ee = ctypes.c_double(); uu = np.zeros(4)
    assert L.vhc_landau(T10.ctypes.data_as(_dp), 1.0, 1, ctypes.byref(ee), uu.ctypes.data_as(_dp)) == 0
    assert find_var(T10, 1.0, True) == []


def test_fluid_at_rest(L):
    """u = 0 exactly: the matching must not fail on u^tau rounding below 1"""
    for e in (0.3, 12.0, 150.0):
        T10 = np.array([e, 0, 0, 0, e / 3, 0, 0, e / 3, 0, e / 3 / 1.7 ** 2])
        ee = ctypes.c_double(); uu = np.zeros(4)
        assert L.vhc_landau(T10.ctypes.data_as(_dp), 1.7, 0, ctypes.byref(ee), uu.ctypes.data_as(_dp)) == 1
        assert abs(ee.value - e) <= 1e-14 * e and abs(uu[0] - 1) <= 1e-15 and np.all(uu[1:] == 0)
