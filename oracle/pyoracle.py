"""ctypes bindings to the oracle (liboracle.so) and to the reference builds
(_ref/libref_*.so).  TEST INFRASTRUCTURE ONLY: imported by tests/, by the
smoke check and by the benchmark's CPU-baseline leg, never by the product.

Both libraries share the canonical state layout described in oracle.h:
18 ghost-inclusive SoA fields, index (k*GY + j)*GX + i.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NF = 18
F_E, F_U, F_PI, F_T, F_PU = 0, 1, 5, 10, 14

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("boost_invariant", ctypes.c_int), ("cartesian", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("eos_kind", ctypes.c_int), ("eos_a", ctypes.c_double), ("eos_n", ctypes.c_int),
        ("eos_e", _dp), ("eos_p", _dp), ("eos_cs2", _dp), ("eos_t", _dp),
        ("etas0", ctypes.c_double), ("etas1", ctypes.c_double), ("etas_tc", ctypes.c_double),
        ("hbarc", ctypes.c_double),
        ("taupi_kind", ctypes.c_int), ("gubser_mirror", ctypes.c_int),
        ("recon", ctypes.c_int), ("minmod_theta", ctypes.c_double), ("taupi_const", ctypes.c_double),
        ("cold_plasma", ctypes.c_int),
    ]


@dataclass
class OracleConfig:
    nx: int
    ny: int
    nz: int = 1
    boost_invariant: bool = True
    cartesian: bool = False
    dx: float = 0.1
    dy: float = 0.1
    dz: float = 0.1
    eos_kind: int = 0          # 0 conformal, 1 table
    eos_a: float = 0.0         # e = a T^4 (fm units) for the conformal EOS
    eos_table: np.ndarray | None = None  # (4, n): e, P, cs2, T in fm units
    etas0: float = 0.08
    etas1: float = 0.0
    etas_tc: float = 0.154
    hbarc: float = 0.19733
    taupi_kind: int = 0        # 0: 1.5 eta/P, 1: 5 eta/(e+P), 2: taupi_const
    taupi_const: float = 0.0
    cold_plasma: bool = False  # shear source without -pi/tau_pi
    gubser_mirror: bool = False
    recon: int = 0             # 0 WENO5, 1 generalized minmod
    minmod_theta: float = 1.1
    _keep: list = field(default_factory=list, repr=False)

    def gdims(self):
        gz = 1 if self.boost_invariant else self.nz + 6
        return self.nx + 6, self.ny + 6, gz

    def to_c(self) -> _Cfg:
        c = _Cfg()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.boost_invariant = int(self.boost_invariant)
        c.cartesian = int(self.cartesian)
        c.dx, c.dy, c.dz = self.dx, self.dy, self.dz
        c.eos_kind, c.eos_a = self.eos_kind, self.eos_a
        if self.eos_kind == 1:
            t = np.ascontiguousarray(self.eos_table, dtype=np.float64)
            self._keep = [t]
            c.eos_n = t.shape[1]
            c.eos_e, c.eos_p, c.eos_cs2, c.eos_t = (t[q].ctypes.data_as(_dp) for q in range(4))
        c.etas0, c.etas1, c.etas_tc, c.hbarc = self.etas0, self.etas1, self.etas_tc, self.hbarc
        c.taupi_kind = self.taupi_kind
        c.gubser_mirror = int(self.gubser_mirror)
        c.recon, c.minmod_theta = self.recon, self.minmod_theta
        c.taupi_const = self.taupi_const
        c.cold_plasma = int(self.cold_plasma)
        return c


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    return ctypes.CDLL(path)


class Oracle:
    """The C restatement of the reference step (liboracle.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = _load(os.path.join(HERE, "liboracle.so"))
            L.vho_create.restype = ctypes.c_void_p
            L.vho_create.argtypes = [ctypes.POINTER(_Cfg)]
            for name in ("vho_destroy", "vho_dims", "vho_set_state", "vho_get_state", "vho_step",
                         "vho_stage_terms", "vho_ns_init", "vho_boundary", "vho_fill_tmunu",
                         "vho_max_temp_gev", "vho_last_iterations", "vho_eos", "vho_con2prim",
                         "vho_is_source", "vho_residual", "vho_ns_pi10", "vho_ns_pi10_cell"):
                getattr(L, name).argtypes = None
            L.vho_destroy.argtypes = [ctypes.c_void_p]
            L.vho_set_state.argtypes = [ctypes.c_void_p, _dp]
            L.vho_get_state.argtypes = [ctypes.c_void_p, _dp]
            L.vho_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
            L.vho_step.restype = ctypes.c_int
            L.vho_stage_terms.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
            L.vho_ns_init.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
            L.vho_boundary.argtypes = [ctypes.c_void_p]
            L.vho_fill_tmunu.argtypes = [ctypes.c_void_p, ctypes.c_double]
            L.vho_max_temp_gev.argtypes = [ctypes.c_void_p]
            L.vho_max_temp_gev.restype = ctypes.c_double
            L.vho_last_iterations.argtypes = [ctypes.c_void_p]
            L.vho_last_iterations.restype = ctypes.c_longlong
            L.vho_eos.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp]
            L.vho_con2prim.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, _dp]
            L.vho_con2prim.restype = ctypes.c_int
            L.vho_is_source.argtypes = [ctypes.c_void_p, ctypes.c_double, _dp, _dp, _dp, ctypes.c_double, _dp]
            L.vho_residual.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
            L.vho_ns_pi10.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp]
            L.vho_ns_pi10_cell.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
            cls._lib = L
        return cls._lib

    def __init__(self, cfg: OracleConfig):
        self.cfg = cfg
        self._c = cfg.to_c()
        self.h = self.lib().vho_create(ctypes.byref(self._c))
        self.gx, self.gy, self.gz = cfg.gdims()
        self.n = self.gx * self.gy * self.gz

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().vho_destroy(self.h)
            self.h = None

    def set_state(self, f: np.ndarray):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(NF, self.n)
        self.lib().vho_set_state(self.h, _ptr(f))

    def get_state(self) -> np.ndarray:
        f = np.zeros((NF, self.n))
        self.lib().vho_get_state(self.h, _ptr(f))
        return f

    def step(self, tau: float, ts: float) -> int:
        return self.lib().vho_step(self.h, tau, ts)

    def stage_terms(self, tau, ts):
        src = np.zeros((10, self.n)); res = np.zeros((10, self.n)); du = np.zeros((16, self.n))
        self.lib().vho_stage_terms(self.h, tau, ts, _ptr(src), _ptr(res), _ptr(du))
        return src, res, du

    def ns_init(self, tau, ts):
        self.lib().vho_ns_init(self.h, tau, ts)

    def ns_pi10(self, tau, ts):
        """2 eta sigma^{mu nu} (10, n) with the step's velocity derivatives"""
        out = np.zeros((10, self.n))
        self.lib().vho_ns_pi10(self.h, tau, ts, _ptr(out))
        return out

    def ns_pi10_cell(self, tau, e, u, du16):
        out = np.zeros(10)
        self.lib().vho_ns_pi10_cell(self.h, tau, e, _ptr(np.ascontiguousarray(u, dtype=np.float64)),
                                    _ptr(np.ascontiguousarray(du16, dtype=np.float64)), _ptr(out))
        return out

    def boundary(self):
        self.lib().vho_boundary(self.h)

    def fill_tmunu(self, tau):
        self.lib().vho_fill_tmunu(self.h, tau)

    def max_temp_gev(self) -> float:
        return self.lib().vho_max_temp_gev(self.h)

    def last_iterations(self) -> int:
        return self.lib().vho_last_iterations(self.h)

    def eos(self, e: float):
        out = np.zeros(6)
        self.lib().vho_eos(self.h, e, _ptr(out))
        return out

    def residual(self, x, prm):
        y = np.zeros(4); J = np.zeros(16)
        self.lib().vho_residual(self.h, _ptr(np.ascontiguousarray(x, dtype=np.float64)),
                                _ptr(np.ascontiguousarray(prm, dtype=np.float64)), _ptr(y), _ptr(J))
        return y, J.reshape(4, 4)


class RefBuild:
    """One compile-time scenario of the reference, built by oracle/Makefile."""

    def __init__(self, variant: str):
        path = os.path.join(HERE, "_ref", f"libref_{variant}.so")
        L = _load(path)
        for name in ("ref_tvdrk2", "ref_tvdrk3"):
            getattr(L, name).argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_stage_terms.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
        L.ref_ns_init.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_eos.argtypes = [ctypes.c_double, _dp]
        L.ref_max_temp_gev.restype = ctypes.c_double
        L.ref_residual.argtypes = [_dp, _dp, _dp, _dp]
        self.L = L
        L.ref_init_grid()
        d = (ctypes.c_int * 10)()
        L.ref_dims(d)
        self.gx, self.gy, self.gz, self.il, self.ir, self.jl, self.jr, self.kl, self.kr, lbi = list(d)
        self.boost_invariant = bool(lbi)
        c = (ctypes.c_double * 5)()
        L.ref_consts(c)
        self.dx, self.dy, self.dz, self.factor, self.gevfm = list(c)
        self.n = self.gx * self.gy * self.gz

    def set_eos_table(self, table):
        """the run-time EOS table (4, n: e, P, cs2, T) of the table-EOS
        builds (libref_window_*.so)"""
        t = np.ascontiguousarray(table, dtype=np.float64)
        self.L.ref_set_eos_table.argtypes = [ctypes.c_int, _dp]
        if self.L.ref_set_eos_table(t.shape[1], _ptr(t)) != 0:
            raise ValueError("bad EOS table")

    def coords(self):
        x = np.zeros(self.n); y = np.zeros(self.n); e = np.zeros(self.n)
        self.L.ref_coords(_ptr(x), _ptr(y), _ptr(e))
        return x, y, e

    def set_state(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(NF, self.n)
        self.L.ref_set_state(_ptr(f))

    def get_state(self):
        f = np.zeros((NF, self.n))
        self.L.ref_get_state(_ptr(f))
        return f

    def step(self, tau, ts):
        self.L.ref_tvdrk2(tau, ts)

    def stage_terms(self, tau, ts):
        src = np.zeros((10, self.n)); res = np.zeros((10, self.n)); du = np.zeros((16, self.n))
        self.L.ref_stage_terms(tau, ts, _ptr(src), _ptr(res), _ptr(du))
        return src, res, du

    def ns_init(self, tau, ts):
        self.L.ref_ns_init(tau, ts)

    def eos(self, e):
        out = np.zeros(6)
        self.L.ref_eos(e, _ptr(out))
        return out

    def max_temp_gev(self):
        return self.L.ref_max_temp_gev()

    def residual(self, x, p):
        y = np.zeros(4); J = np.zeros(16)
        self.L.ref_residual(_ptr(np.ascontiguousarray(x, dtype=np.float64)),
                            _ptr(np.ascontiguousarray(p, dtype=np.float64)), _ptr(y), _ptr(J))
        return y, J.reshape(4, 4)


class RefWrite:
    """The reference's snapshot writers (oracle/ref_write.cpp): NEWEST5's
    write.h (12 doubles per cell) or NEWEST10's (17, and the Navier-Stokes
    snapshot) in one compile-time block."""

    def __init__(self, variant: str):
        L = _load(os.path.join(HERE, "_ref", f"libref_{variant}.so"))
        d = (ctypes.c_int * 9)()
        c = (ctypes.c_double * 4)()
        L.refw_init(d, c)
        L.refw_set_state.argtypes = [_dp, _dp, _dp]
        L.refw_write_xy.argtypes = [ctypes.c_double]
        self.n10 = hasattr(L, "refw_write_ns_xy")
        if self.n10:
            L.refw_write_ns_xy.argtypes = [ctypes.c_double]
        else:
            L.refw_write_full.argtypes = [ctypes.c_double]
        self.L = L
        self.gx, self.gy, self.gz, self.nx, self.ny, self.nz, self.freq, self.freqz, lbi = list(d)
        self.boost_invariant = bool(lbi)
        self.dx, self.dy, self.dz, self.factor = list(c)
        self.n = self.gx * self.gy * self.gz

    def set_state(self, f, pi10=None, nspi=None):
        c = lambda a: None if a is None else _ptr(np.ascontiguousarray(a, dtype=np.float64))
        self.L.refw_set_state(c(f), c(pi10), c(nspi))

    def write(self, which: str, tau: float, workdir: str) -> bytes:
        """the file the reference's writer leaves in workdir/res/"""
        name = ("NStau%2.3ffm.bin" if which == "ns_xy" else "tau%2.3ffm.bin") % tau
        os.makedirs(os.path.join(workdir, "res"), exist_ok=True)
        path = os.path.join(workdir, "res", name)
        if os.path.exists(path):
            os.remove(path)
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            {"xy": lambda: self.L.refw_write_xy(tau), "full": lambda: self.L.refw_write_full(tau),
             "ns_xy": lambda: self.L.refw_write_ns_xy(tau)}[which]()
        finally:
            os.chdir(cwd)
        with open(path, "rb") as fh:
            return fh.read()


class RefNS10:
    """NEWEST10's CalcNS in its default compile-time block, boost invariant
    (oracle/ref_ns10.cpp)."""

    def __init__(self):
        L = _load(os.path.join(HERE, "_ref", "libref_ns10_lbi.so"))
        L.ref10_calc_ns.argtypes = [_dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
        d = (ctypes.c_int * 9)()
        c = (ctypes.c_double * 3)()
        L.ref10_init(d, c)
        self.L = L
        self.gx, self.gy, self.gz, self.il, self.ir, self.jl, self.jr, self.kl, self.kr = list(d)
        self.dx, self.dy, self.factor = list(c)
        self.n = self.gx * self.gy * self.gz

    def calc_ns(self, f, du3, tau, ts):
        """returns nspi + nsPI (11, n) and the du it used (16, n)"""
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(NF, self.n)
        du3 = np.ascontiguousarray(du3, dtype=np.float64).reshape(4, self.n)
        ns = np.zeros((11, self.n)); du = np.zeros((16, self.n))
        self.L.ref10_calc_ns(_ptr(f), _ptr(du3), tau, ts, _ptr(ns), _ptr(du))
        return ns, du


_EIG_FN = ctypes.CFUNCTYPE(ctypes.c_int, _dp, _dp, _dp, _dp, _dp)


def _eig_callback(a, wr, wi, vr, vi):
    """eigenpairs of a real 4x4 matrix (LAPACK dgeev through NumPy) for the
    GSL stand-in of the reference harness"""
    A = np.ctypeslib.as_array(a, shape=(16,)).reshape(4, 4).copy()
    w, v = np.linalg.eig(A)
    w = np.asarray(w, dtype=complex)
    v = np.asarray(v, dtype=complex)
    for i in range(4):
        wr[i] = w[i].real
        wi[i] = w[i].imag
        for j in range(4):
            vr[j * 4 + i] = v[j, i].real
            vi[j * 4 + i] = v[j, i].imag
    return 0


class RefGinit:
    """NEWEST5's Glasma initialisation (ginit.h) in its GINIT block, one
    rank's window of the reference's 10 x 10 layout (oracle/ref_ginit.cpp)."""

    def __init__(self, xcord=4, ycord=4):
        L = _load(os.path.join(HERE, "_ref", "libref_ginit.so"))
        L.ref_ginit_run.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_ginit_eos.argtypes = [ctypes.c_double, _dp]
        L.ref_ginit_e_at_0p4gev.restype = ctypes.c_double
        self._cb = _EIG_FN(_eig_callback)
        L.ref_ginit_set_eig(self._cb)
        d = (ctypes.c_int * 10)()
        c = (ctypes.c_double * 8)()
        L.ref_ginit_init(xcord, ycord, d, c)
        self.L = L
        self.gx, self.gy, self.gz, self.il, self.ir, self.jl, self.jr, self.kl, self.kr, lbi = list(d)
        self.boost_invariant = bool(lbi)
        self.dx, self.dy, self.dz, self.tau0, self.ts, self.x_pos, self.flat, self.gevfm = list(c)
        self.n = self.gx * self.gy * self.gz

    def run(self):
        """ginit at tau0 - ts, then at tau0; returns (state (18, n), x, y, eta)"""
        self.L.ref_ginit_run(self.tau0, self.ts)
        f = np.zeros((NF, self.n)); x = np.zeros(self.n); y = np.zeros(self.n); eta = np.zeros(self.n)
        self.L.ref_ginit_state(_ptr(f), _ptr(x), _ptr(y), _ptr(eta))
        return f, x, y, eta

    def eos(self, e):
        """P, dP/de, T, s of the block's EOS (s95p)"""
        out = np.zeros(4)
        self.L.ref_ginit_eos(e, _ptr(out))
        return out

    def e_at_0p4gev(self):
        return self.L.ref_ginit_e_at_0p4gev()


# ---------------------------------------------------------------- inputs


def grid_coords(gx, gy, gz, dx, dy, dz, boost_invariant):
    """Cell-centre coordinates of the ghost-inclusive grid, centred the way
    the reference centres one rank (NEWEST5/init.h:20-80 with integer
    division of the point count)."""
    nx, ny = gx - 6, gy - 6
    x0 = -((nx // 2) * dx)
    y0 = -((ny // 2) * dy)
    i = np.arange(gx); j = np.arange(gy); k = np.arange(gz)
    X = x0 + (i - 3) * dx
    Y = y0 + (j - 3) * dy
    if boost_invariant:
        Z = np.zeros(gz)
    else:
        nz = gz - 6
        Z = -((nz // 2) * dz) + (k - 3) * dz
    ZZ, YY, XX = np.meshgrid(Z, Y, X, indexing="ij")
    return XX.ravel(), YY.ravel(), ZZ.ravel()


def smooth_state(x, y, z, tau, ts, seed=0, amp=1.0, cartesian=False):
    """A seeded smooth, causal, viscous state on every cell (ghosts
    included): the random-smooth-state fixture of the stage tests."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * math.pi, size=(12,))
    kk = rng.uniform(0.5, 1.4, size=(12,))

    def w(q, a, b):
        return a + b * amp * np.sin(kk[q] * x + ph[q]) * np.cos(kk[(q + 3) % 12] * y + ph[(q + 5) % 12]) \
            * np.cos(0.6 * z + ph[(q + 7) % 12])

    t2 = 1.0 if cartesian else tau * tau
    e = w(0, 12.0, 4.0)
    u1 = w(1, 0.0, 0.3); u2 = w(2, 0.0, 0.25); u3 = w(3, 0.0, 0.08)
    u0 = np.sqrt(1 + u1 * u1 + u2 * u2 + t2 * u3 * u3)
    p = [w(4, 0.0, 0.2), w(5, 0.0, 0.15), w(6, 0.0, 0.1), w(7, 0.0, 0.05), w(8, 0.0, 0.04)]
    tp = 1.0 if cartesian else tau - ts
    pu1, pu2, pu3 = u1 * 0.99, u2 * 1.01, u3 * 0.98
    pu0 = np.sqrt(1 + pu1 ** 2 + pu2 ** 2 + (tp * tp if not cartesian else 1.0) * pu3 ** 2)
    f = np.zeros((NF, x.size))
    f[F_E] = e
    f[F_U:F_U + 4] = [u0, u1, u2, u3]
    f[F_PI:F_PI + 5] = p
    f[F_PU:F_PU + 4] = [pu0, pu1, pu2, pu3]
    return f
