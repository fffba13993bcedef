"""The algorithm of the GPU freeze-out (vh_freezeout_*_device,
vh_cooper_frye_*_device) run on the host through libvh_check.so, which
exposes the same __host__ __device__ functions the kernels call: per-cube
counts from the signs of T - T_fo, their exclusive scan and each cube's
elements written from its offset, in any order of the cubes, give the host
functions' elements exactly; the quadrature K0, K1 of the boost-invariant
spectrum against SciPy; the device entry points' argument checks (which
return before any CUDA call)."""
import ctypes
import itertools

import numpy as np
import pytest
from scipy import special

from viral_b200 import _abi as A
from viral_b200 import build
from viral_b200.hydro import cooper_frye_2d, cooper_frye_3d, freezeout_2d, freezeout_3d

_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_longlong)


@pytest.fixture(scope="module")
def L():
    lib = ctypes.CDLL(build.build_check())
    lib.vhc_fo_emulate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp,
                                   _dp, ctypes.c_double, _lp, _dp, ctypes.c_longlong]
    lib.vhc_fo_emulate.restype = ctypes.c_longlong
    lib.vhc_bessel_k01e.argtypes = [ctypes.c_double, _dp]
    lib.vhc_bessel_k01e.restype = None
    lib.vhc_cf2_term.argtypes = [_dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.vhc_cf2_term.restype = ctypes.c_double
    lib.vhc_kuhn_simplex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.vhc_kuhn_simplex.restype = None
    return lib


def ptr(a):
    return a.ctypes.data_as(_dp)


def test_kuhn_simplices_follow_the_axis_permutations(L):
    for m in (3, 4):
        for s, perm in enumerate(itertools.permutations(range(m))):
            v = (ctypes.c_int * 5)()
            L.vhc_kuhn_simplex(s, m, v)
            want, bits = [0], 0
            for a in perm:
                bits |= 1 << a
                want.append(bits)
            assert list(v)[:m + 1] == want


def fields_2d(nx, ny, dx, dy, seed):
    """a hot spot with flow and a rough surface: every cut pattern of the
    cube's tetrahedra, and corners exactly at T_fo"""
    gx, gy = nx + 6, ny + 6
    X = -(nx // 2) * dx + (np.arange(gx) - 3) * dx
    Y = -(ny // 2) * dy + (np.arange(gy) - 3) * dy
    YY, XX = np.meshgrid(Y, X, indexing="ij")
    x, y = XX.ravel(), YY.ravel()
    rng = np.random.default_rng(seed)
    T0 = 0.3 * np.exp(-(x * x + 0.5 * y * y) / 2) + 0.02 * rng.standard_normal(x.size)
    T1 = 0.9 * T0 + 0.02 * rng.standard_normal(x.size)
    T0[::17] = 0.15  # on the isotherm: counted as the cold side
    u = lambda s: np.stack([np.sqrt(1 + s * s * (x * x + y * y)), s * x, s * y])
    return T0, T1, u(0.3), u(0.35)


def emulate(L, D, dims, d, tau0, tau1, T0, T1, u0, u1, tfo, perm, cap):
    nx, ny, nz = dims
    out = np.zeros((max(cap, 1), 9 if D == 3 else 12))
    u0, u1 = np.ascontiguousarray(u0), np.ascontiguousarray(u1)
    p = np.ascontiguousarray(perm, dtype=np.int64)
    total = L.vhc_fo_emulate(D, nx, ny, nz, d[0], d[1], d[2], tau0, tau1, ptr(T0), ptr(T1), ptr(u0), ptr(u1), tfo,
                             p.ctypes.data_as(_lp), ptr(out), cap)
    return total, out[:max(total, 0)]


def test_device_algorithm_gives_the_host_elements_2d(L):
    nx, ny, dx, dy = 23, 19, 0.1, 0.15
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 1)
    host = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, T0, T1, u0, u1, 0.15)
    assert len(host) > 200
    nc = (nx - 1) * (ny - 1)
    for perm in (np.arange(nc), np.arange(nc)[::-1], np.random.default_rng(2).permutation(nc)):
        total, el = emulate(L, 3, (nx, ny, 1), (dx, dy, 0.0), 1.0, 1.1, T0, T1, u0, u1, 0.15, perm, len(host))
        assert total == len(host)  # and every cube emitted its count (else -1)
        assert np.array_equal(el, host)


def test_device_algorithm_gives_the_host_elements_3d(L):
    nx, ny, nz, dx, dy, dz = 9, 8, 7, 0.1, 0.12, 0.2
    gx, gy, gz = nx + 6, ny + 6, nz + 6
    rng = np.random.default_rng(3)
    n = gx * gy * gz
    T0 = 0.15 + 0.04 * rng.standard_normal(n)
    T1 = 0.15 + 0.04 * rng.standard_normal(n)
    T0[::13] = 0.15
    u0 = np.vstack([1 + rng.random(n), 0.3 * rng.standard_normal((3, n))])
    u1 = np.vstack([1 + rng.random(n), 0.3 * rng.standard_normal((3, n))])
    host = freezeout_3d(nx, ny, nz, dx, dy, dz, 0.8, 0.85, T0, T1, u0, u1, 0.15)
    assert len(host) > 5000  # every one of the 24 simplices' cut patterns occurs
    nc = (nx - 1) * (ny - 1) * (nz - 1)
    for perm in (np.arange(nc)[::-1], np.random.default_rng(4).permutation(nc)):
        total, el = emulate(L, 4, (nx, ny, nz), (dx, dy, dz), 0.8, 0.85, T0, T1, u0, u1, 0.15, perm, len(host))
        assert total == len(host)
        assert np.array_equal(el, host)


def test_device_algorithm_respects_the_capacity(L):
    nx, ny, dx, dy = 15, 15, 0.1, 0.1
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 5)
    host = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, T0, T1, u0, u1, 0.15)
    cap = len(host) // 3
    nc = (nx - 1) * (ny - 1)
    out = np.full((cap + 4, 9), 7.0)  # 4 guard rows that must stay untouched
    p = np.random.default_rng(6).permutation(nc).astype(np.int64)
    total = L.vhc_fo_emulate(3, nx, ny, 1, dx, dy, 0.0, 1.0, 1.1, ptr(T0), ptr(T1), ptr(np.ascontiguousarray(u0)),
                             ptr(np.ascontiguousarray(u1)), 0.15, p.ctypes.data_as(_lp), ptr(out), cap)
    assert total == len(host)
    assert np.array_equal(out[:cap], host[:cap]) and np.all(out[cap:] == 7.0)


def test_quadrature_bessel_functions(L):
    z = np.logspace(-6, 3, 400)
    got = np.zeros((z.size, 2))
    for i, zi in enumerate(z):
        L.vhc_bessel_k01e(zi, ptr(got[i]))
    assert np.abs(got[:, 0] / special.k0e(z) - 1).max() <= 5e-15
    assert np.abs(got[:, 1] / special.k1e(z) - 1).max() <= 5e-15


def test_spectrum_against_scipy_bessel_functions():
    """the boost-invariant spectrum (quadrature K0, K1 in scaled form) against
    the same sum written here with SciPy's K0, K1"""
    nx, ny, dx, dy = 31, 31, 0.2, 0.2
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 7)
    el = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, np.abs(T0), np.abs(T1), u0, u1, 0.15)
    tfo, m, g = 0.15, 0.7, 3.0
    pt, phi = np.array([0.0, 0.3, 1.0, 2.5]), np.array([0.0, 0.7, 2.0])
    got = cooper_frye_2d(el, tfo, m, g, pt, phi)
    want = np.zeros_like(got)
    for a, p in enumerate(pt):
        mt = np.sqrt(m * m + p * p)
        arg = mt * el[:, 6] / tfo
        for b, f in enumerate(phi):
            px, py = p * np.cos(f), p * np.sin(f)
            terms = (2 * mt * special.k1(arg) * el[:, 3] + 2 * special.k0(arg) * (px * el[:, 4] + py * el[:, 5])) \
                * np.exp((px * el[:, 7] + py * el[:, 8]) / tfo)
            want[a, b] = g / (8 * np.pi ** 3) * terms.sum()
    assert np.allclose(got, want, rtol=1e-13, atol=0)


def test_spectrum_stays_finite_at_large_momentum():
    """p_T u_perp / T far above the exponent range of a double: the scaled
    Bessel functions keep the term finite (the product K1(a) e^b would be
    0 times infinity)"""
    el = np.zeros((1, 9))
    el[0, 3], el[0, 6], el[0, 7] = 1.0, np.sqrt(1 + 4.0), 2.0  # u^x = 2
    sp = cooper_frye_2d(el, 0.15, 0.14, 1.0, [60.0, 120.0], [0.0])
    assert np.all(np.isfinite(sp)) and np.all(sp > 0)


def test_device_entry_points_check_arguments_first():
    """bad arguments return VH_E_ARG before any CUDA call (so also here,
    without a GPU); the pointers are never dereferenced"""
    Lb = A.lib()
    cnt = ctypes.c_longlong(-5)
    fake = 16  # a non-null device address that the checks must not use
    assert Lb.vh_freezeout_2d_device(1, 8, 0.1, 0.1, 1.0, 1.1, fake, fake, fake, fake, 0.15, None, 0,
                                     ctypes.byref(cnt), None) == A.E_ARG
    assert Lb.vh_freezeout_2d_device(8, 8, 0.1, 0.1, 1.1, 1.0, fake, fake, fake, fake, 0.15, None, 0,
                                     ctypes.byref(cnt), None) == A.E_ARG
    assert Lb.vh_freezeout_2d_device(8, 8, 0.1, 0.1, 1.0, 1.1, fake, fake, fake, fake, 0.15, None, 4,
                                     ctypes.byref(cnt), None) == A.E_ARG  # cap without out
    assert Lb.vh_freezeout_3d_device(8, 8, 1, 0.1, 0.1, 0.1, 1.0, 1.1, fake, fake, fake, fake, 0.15, None, 0,
                                     ctypes.byref(cnt), None) == A.E_ARG
    assert Lb.vh_freezeout_3d_device(8, 8, 8, 0.1, 0.1, 0.1, 1.0, 1.1, None, fake, fake, fake, 0.15, None, 0,
                                     ctypes.byref(cnt), None) == A.E_ARG
    assert cnt.value == -5
    pt, phi, out = np.array([0.0, 1.0]), np.array([0.0]), np.zeros(2)
    # a massless hadron at p_T = 0 in the boost-invariant form; t_fo <= 0;
    # a negative count
    assert Lb.vh_cooper_frye_2d_device(fake, 10, 0.15, 0.0, 1.0, ptr(pt), 2, ptr(phi), 1, ptr(out), None) == A.E_ARG
    assert Lb.vh_cooper_frye_2d_device(fake, 10, 0.0, 0.1, 1.0, ptr(pt), 2, ptr(phi), 1, ptr(out), None) == A.E_ARG
    assert Lb.vh_cooper_frye_3d_device(fake, -1, 0.15, 0.1, 1.0, 0.0, ptr(pt), 2, ptr(phi), 1, ptr(out),
                                       None) == A.E_ARG
    assert Lb.vh_cooper_frye_3d_device(fake, 10, 0.15, 0.1, 1.0, float("nan"), ptr(pt), 2, ptr(phi), 1, ptr(out),
                                       None) == A.E_ARG


def test_host_spectra_refuse_a_massless_hadron_at_zero_momentum():
    el = np.zeros((1, 9))
    el[0, 3], el[0, 6] = 1.0, 1.0
    with pytest.raises(RuntimeError):
        cooper_frye_2d(el, 0.15, 0.0, 1.0, [0.0, 0.5], [0.0])
    # 3+1D: p^mu dSigma_mu vanishes with m_T, no limit to take
    el3 = np.zeros((1, 12))
    el3[0, 0], el3[0, 4], el3[0, 8] = 1.0, 1.0, 1.0
    assert cooper_frye_3d(el3, 0.15, 0.0, 1.0, 0.0, [0.0], [0.0])[0, 0] == 0.0


def test_device_wrappers_want_cuda_tensors():
    """the Python wrappers of the device forms take CUDA tensors and check
    their sizes before any call (so also here, without a GPU)"""
    import torch
    from viral_b200.hydro import _cuda_f64, cooper_frye_2d_device, freezeout_2d_device
    n = 14 * 14
    with pytest.raises(TypeError):
        freezeout_2d_device(8, 8, 0.1, 0.1, 1.0, 1.1, np.zeros(n), np.zeros(n), np.zeros((3, n)), np.zeros((3, n)), 0.15)
    with pytest.raises(TypeError):
        cooper_frye_2d_device(torch.zeros((4, 9)), 0.15, 0.1, 1.0, [0.5], [0.0])
    with pytest.raises(TypeError):
        _cuda_f64(torch.zeros(n), 0, n)
