"""Local adjoints of the 3+1D Milne step (every evolved field, the eta
direction, its Christoffel terms), checked against central finite
differences on the CPU through libvh_check.so, which compiles the same
__host__ __device__ functions the 3+1D adjoint kernels run: the pi closure,
the flux quantities along x, y and eta, the geometric and shear sources, and
the root of the four-unknown conserved-to-primitive system."""
import ctypes

import numpy as np
import pytest

from test_adjoint_cpu import _dp, P, arr, cfgs, check_vjp, fd
from viral_b200 import _abi as A
from viral_b200 import build


@pytest.fixture(scope="module")
def L():
    lib = ctypes.CDLL(build.build_check())
    cfgp = ctypes.POINTER(A.VhConfig)
    d = ctypes.c_double
    sig = {
        "vhc_pi_dep": ([_dp, _dp, d, _dp], None),
        "vhc_pi_dep_vjp": ([_dp, _dp, d, _dp, _dp, _dp], None),
        "vhc_cell_q3": ([cfgp, ctypes.c_int, d, _dp, ctypes.c_int, _dp], None),
        "vhc_cell_q3_vjp": ([cfgp, ctypes.c_int, d, _dp, ctypes.c_int, _dp, _dp], None),
        "vhc_src3": ([cfgp, d, d, _dp, _dp, _dp, _dp], None),
        "vhc_src3_vjp": ([cfgp, d, d, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp], None),
        "vhc_con2prim4": ([cfgp, _dp, _dp, d, _dp], ctypes.c_int),
        "vhc_c2p_ift_vjp4": ([cfgp, _dp, _dp, d, _dp, _dp, _dp, _dp], ctypes.c_int),
        "vhc_eos_d": ([cfgp, d, _dp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


def velocity(rng, t2, scale=0.5):
    u1, u2 = rng.normal(scale=scale, size=2)
    u3 = rng.normal(scale=scale) / np.sqrt(t2)
    return np.array([np.sqrt(1 + u1 * u1 + u2 * u2 + t2 * u3 * u3), u1, u2, u3])


def test_pi_closure_vjp(L):
    rng = np.random.default_rng(21)
    for t2 in (0.36, 1.0, 6.25):
        for trial in range(4):
            z = np.concatenate([velocity(rng, t2), rng.normal(scale=0.3, size=5)])

            def f(zz):
                out = arr(5)
                L.vhc_pi_dep(P(zz[:4]), P(zz[4:]), t2, out.ctypes.data_as(_dp))
                return out
            J = fd(f, z, 1e-7)
            db = rng.normal(size=5)
            ub, pb = arr(4), arr(5)
            L.vhc_pi_dep_vjp(P(z[:4]), P(z[4:]), t2, P(db), ub.ctypes.data_as(_dp), pb.ctypes.data_as(_dp))
            check_vjp(J, np.concatenate([ub, pb]), db, 1e-6)


def cell_x3(rng, e_scale, tau):
    e = e_scale * rng.uniform(0.5, 2.0)
    u = velocity(rng, tau * tau, 0.6)
    p = rng.normal(scale=0.05 * e, size=5)
    T = rng.normal(scale=e, size=4)
    return np.concatenate([[e], u, p, T])


@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("interior", [0, 1])
def test_cell_q3_vjp(L, direction, interior):
    rng = np.random.default_rng(30 + direction + 3 * interior)
    tau = 1.3
    for name, cfg in cfgs():
        c = cfg.to_c()
        for e_scale in (0.05, 3.0, 80.0):
            x = cell_x3(rng, e_scale, tau)

            def f(xx):
                q = arr(19)
                L.vhc_cell_q3(ctypes.byref(c), direction, tau, P(xx), interior, q.ctypes.data_as(_dp))
                return q
            J = fd(f, x, 1e-7)
            qb = rng.normal(size=19)
            xb = arr(14)
            L.vhc_cell_q3_vjp(ctypes.byref(c), direction, tau, P(x), interior, P(qb), xb.ctypes.data_as(_dp))
            check_vjp(J, xb, qb, 2e-6)


@pytest.mark.parametrize("which", ["table", "conformal", "const_taupi"])
def test_src3_vjp(L, which):
    rng = np.random.default_rng(41 if which == "table" else 42)
    cfg = dict(cfgs())[which]
    tau = 0.9
    for e in (0.3, 2.0, 9.0, 60.0):  # across the eta/s kink at T = 0.154 GeV
        for trial in range(3):
            c = cfg.to_c()
            u = velocity(rng, tau * tau, 0.4)
            z = np.concatenate([[e], u, rng.normal(scale=0.03 * e, size=5), rng.normal(scale=0.5, size=16),
                                [cfg.etas0, cfg.etas1]])

            def f(zz):
                c.etas0, c.etas1 = zz[26], zz[27]
                out = arr(9)
                L.vhc_src3(ctypes.byref(c), tau, zz[0], P(zz[1:5]), P(zz[5:10]), P(zz[10:26]),
                           out.ctypes.data_as(_dp))
                return out
            J = fd(f, z, 1e-7)
            c.etas0, c.etas1 = cfg.etas0, cfg.etas1
            ob = rng.normal(size=9)
            ob[1] = ob[2] = 0.0  # no x and y geometric sources
            eb = ctypes.c_double(0.0)
            ub, pb, dub, cb = arr(4), arr(5), arr(16), arr(2)
            L.vhc_src3_vjp(ctypes.byref(c), tau, z[0], P(z[1:5]), P(z[5:10]), P(z[10:26]), P(ob),
                           ctypes.byref(eb), ub.ctypes.data_as(_dp), pb.ctypes.data_as(_dp),
                           dub.ctypes.data_as(_dp), cb.ctypes.data_as(_dp))
            got = np.concatenate([[eb.value], ub, pb, dub, cb])
            check_vjp(J, got, ob, 5e-6)


def conserved(L, c, e, u, p, tau):
    """T^{tau mu} of (e, u^mu, pi) with the closure's pi^{tau mu}"""
    t2 = tau * tau
    ed = arr(4)
    L.vhc_eos_d(ctypes.byref(c), e, ed.ctypes.data_as(_dp))
    Pp = ed[0]
    d = arr(5)
    L.vhc_pi_dep(P(u), P(p), t2, d.ctypes.data_as(_dp))
    return np.array([(e + Pp) * u[0] * u[0] - Pp + d[0], (e + Pp) * u[0] * u[1] + d[1],
                     (e + Pp) * u[0] * u[2] + d[2], (e + Pp) * u[0] * u[3] + d[3]])


@pytest.mark.parametrize("which", ["table", "conformal", "const_taupi"])
def test_con2prim4_ift_vjp(L, which):
    rng = np.random.default_rng(47)
    cfg = dict(cfgs())[which]
    c = cfg.to_c()
    tau = 1.1
    for e in (0.2, 5.0, 50.0):
        for trial in range(3):
            u = velocity(rng, tau * tau, 0.6)
            p = rng.normal(scale=0.02 * e, size=5)
            theta = np.concatenate([conserved(L, c, e, u, p, tau), p])

            def root(th):
                x = np.array([e, u[1], u[2], u[3]])
                it = L.vhc_con2prim4(ctypes.byref(c), P(th[:4]), P(th[4:]), tau, x.ctypes.data_as(_dp))
                assert it >= 0
                return x
            x = root(theta)
            assert abs(x[0] - e) <= 1e-10 * e and np.max(np.abs(x[1:] - u[1:])) <= 1e-10
            J = fd(root, theta, 1e-7)
            xb = rng.normal(size=4)
            Tb, pb = arr(4), arr(5)
            ok = L.vhc_c2p_ift_vjp4(ctypes.byref(c), P(theta[:4]), P(theta[4:]), tau, P(x), P(xb),
                                    Tb.ctypes.data_as(_dp), pb.ctypes.data_as(_dp))
            assert ok == 0
            check_vjp(J, np.concatenate([Tb, pb]), xb, 2e-6)
