"""Local adjoints of the step, checked against central finite differences on
the CPU.  libvh_check.so exposes the same __host__ __device__ functions the
GPU kernels run (WENO face states, per-cell flux quantities, the 2+1D
source, the conserved-to-primitive root and the momentum anisotropy), so a
vector-Jacobian product that passes here is the one the adjoint kernels use.
"""
import ctypes

import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200 import build
from viral_b200 import configs as C
from viral_b200.hydro import Config

_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def L():
    lib = ctypes.CDLL(build.build_check())
    cfgp = ctypes.POINTER(A.VhConfig)
    sig = {
        "vhc_weno_lr": [_dp, _dp, _dp],
        "vhc_weno_lr_vjp": [_dp, ctypes.c_double, ctypes.c_double, _dp],
        "vhc_cell_q": [cfgp, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int, _dp],
        "vhc_cell_q_vjp": [cfgp, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int, _dp, _dp],
        "vhc_src2d": [cfgp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp],
        "vhc_src2d_vjp": [cfgp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp],
        "vhc_con2prim": [cfgp, _dp, _dp, ctypes.c_double, _dp],
        "vhc_c2p_ift_vjp": [cfgp, _dp, _dp, ctypes.c_double, _dp, _dp, _dp, _dp],
        "vhc_eos_d": [cfgp, ctypes.c_double, _dp],
        "vhc_obs_cell": [cfgp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                         ctypes.c_double, _dp],
        "vhc_obs_cell_vjp": [cfgp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, _dp],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int if name in ("vhc_con2prim", "vhc_c2p_ift_vjp") else None
    return lib


def P(a):
    """pointer to a float64 array (the pointer keeps the array alive); the
    array itself when it is already contiguous float64, so outputs land in it"""
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def arr(n):
    return np.zeros(n, dtype=np.float64)


def cfgs():
    """conformal and tabulated EOS; the three tau_pi forms; eta/s with a T kink"""
    a = C.glauber_config(nx=8, ny=8, boost_invariant=True, etas0=0.08, etas1=1.0)
    b = Config(nx=8, ny=8, eos_kind=A.EOS_CONFORMAL, etas0=0.2, etas1=0.5, etas_tc=0.154,
               taupi_kind=A.TAUPI_5_ETA_OVER_EPP)
    c = C.bjorken_config(nx=8, ny=8)  # tau_pi a constant 0.01 fm/c
    return [("table", a), ("conformal", b), ("const_taupi", c)]


def fd(f, x, h):
    """central differences of a vector function: J[:, k]"""
    x = np.array(x, dtype=np.float64)
    cols = []
    for k in range(len(x)):
        xp = x.copy(); xm = x.copy()
        hk = h * max(1.0, abs(x[k]))
        xp[k] += hk; xm[k] -= hk
        cols.append((f(xp) - f(xm)) / (2 * hk))
    return np.stack(cols, axis=1)


def check_vjp(J_fd, vjp, ybar, rtol):
    got = vjp
    want = ybar @ J_fd
    scale = max(np.max(np.abs(want)), 1e-300)
    assert np.max(np.abs(got - want)) <= rtol * scale, (got, want)


def test_weno_vjp(L):
    rng = np.random.default_rng(1)
    for trial in range(20):
        q = rng.normal(size=5) * (10 ** rng.uniform(-3, 2))
        if trial % 4 == 0:
            q = np.array([1.0, 1.1, 1.3, 1.2, 0.9]) * 7.0  # smooth and non-monotone
        def f(qq):
            l = ctypes.c_double(); r = ctypes.c_double()
            L.vhc_weno_lr(P(qq), ctypes.byref(l), ctypes.byref(r))
            return np.array([l.value, r.value])
        J = fd(f, q, 1e-6)
        for lb, rb in ((1.0, 0.0), (0.0, 1.0), (0.3, -1.7)):
            qb = arr(5)
            L.vhc_weno_lr_vjp(P(q), lb, rb, P(qb))
            check_vjp(J, qb, np.array([lb, rb]), 1e-6)


def cell_x(rng, e_scale):
    e = e_scale * rng.uniform(0.5, 2.0)
    u1, u2 = rng.normal(scale=0.6, size=2)
    u0 = np.sqrt(1 + u1 * u1 + u2 * u2)
    p = rng.normal(scale=0.05 * e, size=3)
    T = rng.normal(scale=e, size=3)
    return np.array([e, u0, u1, u2, p[0], p[1], p[2], T[0], T[1], T[2]])


@pytest.mark.parametrize("direction", [0, 1])
@pytest.mark.parametrize("interior", [0, 1])
def test_cell_q_vjp(L, direction, interior):
    rng = np.random.default_rng(10 + direction + 2 * interior)
    for name, cfg in cfgs():
        c = cfg.to_c()
        for e_scale in (0.05, 3.0, 80.0):
            x = cell_x(rng, e_scale)
            tau = 1.3
            def f(xx):
                q = arr(13)
                L.vhc_cell_q(ctypes.byref(c), direction, tau, P(xx), interior, q.ctypes.data_as(_dp))
                return q
            J = fd(f, x, 1e-7)
            qb = rng.normal(size=13)
            xb = arr(10)
            L.vhc_cell_q_vjp(ctypes.byref(c), direction, tau, x.ctypes.data_as(_dp), interior,
                             qb.ctypes.data_as(_dp), xb.ctypes.data_as(_dp))
            check_vjp(J, xb, qb, 2e-6)


def src_inputs(rng, e):
    u1, u2 = rng.normal(scale=0.4, size=2)
    u0 = np.sqrt(1 + u1 * u1 + u2 * u2)
    p = rng.normal(scale=0.03 * e, size=3)
    du = rng.normal(scale=0.5, size=9)
    return np.array([e, u0, u1, u2, *p, *du])


@pytest.mark.parametrize("which", ["table", "conformal", "const_taupi"])
def test_src2d_vjp(L, which):
    rng = np.random.default_rng(3 if which == "table" else 4)
    cfg = dict(cfgs())[which]
    for e in (0.3, 2.0, 9.0, 60.0):  # across the eta/s kink at T = 0.154 GeV
        for trial in range(3):
            c = cfg.to_c()
            z = src_inputs(rng, e)
            z = np.concatenate([z, [cfg.etas0, cfg.etas1]])
            tau = 0.9
            def f(zz):
                c.etas0, c.etas1 = zz[16], zz[17]
                out = arr(4)
                L.vhc_src2d(ctypes.byref(c), tau, zz[0], np.ascontiguousarray(zz[1:4]).ctypes.data_as(_dp),
                            np.ascontiguousarray(zz[4:7]).ctypes.data_as(_dp),
                            np.ascontiguousarray(zz[7:16]).ctypes.data_as(_dp), out.ctypes.data_as(_dp))
                return out
            J = fd(f, z, 1e-7)
            c.etas0, c.etas1 = cfg.etas0, cfg.etas1
            ob = rng.normal(size=4)
            eb = ctypes.c_double(0.0)
            ub, pb, dub, cb = arr(3), arr(3), arr(9), arr(2)
            L.vhc_src2d_vjp(ctypes.byref(c), tau, z[0], z[1:4].copy().ctypes.data_as(_dp),
                            z[4:7].copy().ctypes.data_as(_dp), z[7:16].copy().ctypes.data_as(_dp),
                            ob.ctypes.data_as(_dp), ctypes.byref(eb), ub.ctypes.data_as(_dp),
                            pb.ctypes.data_as(_dp), dub.ctypes.data_as(_dp), cb.ctypes.data_as(_dp))
            got = np.concatenate([[eb.value], ub, pb, dub, cb])
            check_vjp(J, got, ob, 5e-6)


@pytest.mark.parametrize("which", ["table", "conformal", "const_taupi"])
def test_con2prim_ift_vjp(L, which):
    rng = np.random.default_rng(7)
    cfg = dict(cfgs())[which]
    c = cfg.to_c()
    tau = 1.1
    for e in (0.2, 5.0, 50.0):
        for trial in range(3):
            u1, u2 = rng.normal(scale=0.7, size=2)
            u0 = np.sqrt(1 + u1 * u1 + u2 * u2)
            p = rng.normal(scale=0.02 * e, size=3)
            # conserved values of (e, u, pi)
            ed = arr(4)
            L.vhc_eos_d(ctypes.byref(c), e, ed.ctypes.data_as(_dp))
            Pp = ed[0]
            ptx = (p[0] * u1 + p[2] * u2) / u0
            pty = (p[2] * u1 + p[1] * u2) / u0
            ptt = (u1 * u1 * p[0] + 2 * u1 * u2 * p[2] + u2 * u2 * p[1]) / (u0 * u0)
            T = np.array([(e + Pp) * u0 * u0 - Pp + ptt, (e + Pp) * u0 * u1 + ptx, (e + Pp) * u0 * u2 + pty])
            theta = np.concatenate([T, p])
            def root(th):
                x = np.array([e, u1, u2])
                it = L.vhc_con2prim(ctypes.byref(c), np.ascontiguousarray(th[:3]).ctypes.data_as(_dp),
                                    np.ascontiguousarray(th[3:]).ctypes.data_as(_dp), tau, x.ctypes.data_as(_dp))
                assert it >= 0
                return x
            x = root(theta)
            assert abs(x[0] - e) <= 1e-10 * e
            J = fd(root, theta, 1e-7)
            xb = rng.normal(size=3)
            Tb, pb = arr(3), arr(3)
            ok = L.vhc_c2p_ift_vjp(ctypes.byref(c), theta[:3].copy().ctypes.data_as(_dp),
                                   theta[3:].copy().ctypes.data_as(_dp), tau, x.ctypes.data_as(_dp),
                                   xb.ctypes.data_as(_dp), Tb.ctypes.data_as(_dp), pb.ctypes.data_as(_dp))
            assert ok == 0
            check_vjp(J, np.concatenate([Tb, pb]), xb, 2e-6)


@pytest.mark.parametrize("which", ["table", "conformal", "const_taupi"])
def test_eos_derivative(L, which):
    cfg = dict(cfgs())[which]
    c = cfg.to_c()
    for e in (0.01, 0.37, 4.2, 77.0):
        d = arr(4); dp = arr(4); dm = arr(4)
        L.vhc_eos_d(ctypes.byref(c), e, d.ctypes.data_as(_dp))
        h = 1e-7 * e
        L.vhc_eos_d(ctypes.byref(c), e + h, dp.ctypes.data_as(_dp))
        L.vhc_eos_d(ctypes.byref(c), e - h, dm.ctypes.data_as(_dp))
        assert abs((dp[0] - dm[0]) / (2 * h) - d[1]) <= 1e-6 * abs(d[1])
        assert abs((dp[2] - dm[2]) / (2 * h) - d[3]) <= 1e-6 * abs(d[3])


def test_observable_vjp(L):
    rng = np.random.default_rng(9)
    cfg = dict(cfgs())["table"]
    c = cfg.to_c()
    N, D = 0.7, 11.0
    for e in (0.5, 8.0):
        x = np.array([e, *rng.normal(scale=0.5, size=2), *rng.normal(scale=0.05 * e, size=2)])
        def f(xx):
            o = arr(2)
            L.vhc_obs_cell(ctypes.byref(c), xx[0], xx[1], xx[2], xx[3], xx[4], o.ctypes.data_as(_dp))
            return np.array([(N + o[0]) / (D + o[1])])
        J = fd(f, x, 1e-7)
        # the cell's own numerator and denominator are part of the totals
        o = arr(2)
        L.vhc_obs_cell(ctypes.byref(c), *x, o.ctypes.data_as(_dp))
        g = arr(5)
        L.vhc_obs_cell_vjp(ctypes.byref(c), x[0], x[1], x[2], N + o[0], D + o[1], g.ctypes.data_as(_dp))
        check_vjp(J, g, np.array([1.0]), 1e-6)
