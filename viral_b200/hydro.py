"""Python handle over the C ABI (include/vh.h), mirroring the reference's
driver surface: initialise from a profile, evolve per step, read the
conserved and primitive arrays, maximum temperature, snapshot writers
(NEWEST5/main.cpp:90-223, init.h:556, time.h:333, utils.h:263, write.h).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

HBARC = 0.19733
A_QGP = math.pi ** 2 * (16 + 31.5) / 90  # e = a T^4 (fm units)

F_E, F_U, F_PI, F_T, F_PU = 0, 1, 5, 10, 14


@dataclass
class Config:
    nx: int
    ny: int
    nz: int = 1
    boost_invariant: bool = True
    coords: int = A.COORD_MILNE
    precision: int = A.PREC_FP64
    recon: int = A.RECON_WENO5
    dx: float = 0.1
    dy: float = 0.1
    dz: float = 0.1
    tau0: float = 0.6
    dtau: float = 0.02
    eos_kind: int = A.EOS_CONFORMAL
    eos_a: float = A_QGP
    eos_table: np.ndarray | None = None  # (4, n): e, P, cs2, T (fm units)
    etas0: float = 0.08
    etas1: float = 0.0
    etas_tc: float = 0.154
    hbarc: float = HBARC
    taupi_kind: int = A.TAUPI_15_ETA_OVER_P
    gubser_mirror: bool = False
    minmod_theta: float = 1.1
    taupi_const: float = 0.0  # tau_pi (fm/c) with TAUPI_CONST
    cold_plasma: bool = False  # the shear source without -pi/tau_pi (COLDPLASMA test)
    _keep: list = field(default_factory=list, repr=False)

    def gdims(self):
        return self.nx + 6, self.ny + 6, (1 if self.boost_invariant else self.nz + 6)

    def to_c(self) -> A.VhConfig:
        c = A.VhConfig()
        c.coords, c.precision, c.recon = self.coords, self.precision, self.recon
        c.nx, c.ny, c.nz = self.nx, self.ny, (1 if self.boost_invariant else self.nz)
        c.boost_invariant = int(self.boost_invariant)
        c.dx, c.dy, c.dz = self.dx, self.dy, self.dz
        c.tau0, c.dtau = self.tau0, self.dtau
        c.eos_kind, c.eos_a = self.eos_kind, self.eos_a
        if self.eos_kind == A.EOS_TABLE:
            t = np.ascontiguousarray(self.eos_table, dtype=np.float64)
            self._keep = [t]
            c.eos_n = t.shape[1]
            c.eos_e, c.eos_p, c.eos_cs2, c.eos_t = (A.ptr(t[q]) for q in range(4))
        c.etas0, c.etas1, c.etas_tc, c.hbarc = self.etas0, self.etas1, self.etas_tc, self.hbarc
        c.taupi_kind = self.taupi_kind
        c.gubser_mirror = int(self.gubser_mirror)
        c.minmod_theta = self.minmod_theta
        c.taupi_const = self.taupi_const
        c.cold_plasma = int(self.cold_plasma)
        return c


class Hydro:
    """One event on the GPU behind a vh_handle."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self._c = cfg.to_c()
        h = ctypes.c_void_p()
        A.check(A.lib().vh_create(ctypes.byref(self._c), ctypes.byref(h)))
        self.h = h
        self.gx, self.gy, self.gz = cfg.gdims()
        self.n = self.gx * self.gy * self.gz

    def close(self):
        if getattr(self, "h", None):
            A.lib().vh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, code):
        A.check(code, self.h)

    # ---- state
    def set_state(self, f: np.ndarray, tau: float):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(A.NFIELDS, self.n)
        self._chk(A.lib().vh_set_state(self.h, A.ptr(f), tau))

    def get_state(self) -> np.ndarray:
        f = np.empty((A.NFIELDS, self.n))
        self._chk(A.lib().vh_get_state(self.h, A.ptr(f)))
        return f

    def get_primitive(self) -> dict:
        """e, P, T (n,), u (4, n), pi (10, n: tt tx ty te xx xy xe yy ye ee)"""
        e, P, T = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        u, pi = np.zeros((4, self.n)), np.zeros((10, self.n))
        self._chk(A.lib().vh_get_primitive(self.h, A.ptr(e), A.ptr(P), A.ptr(T), A.ptr(u), A.ptr(pi)))
        return dict(e=e, P=P, T=T, u=u, pi=pi)

    def get_conserved(self) -> np.ndarray:
        """the reference's Var (10, n): tau T^{tau mu}, pi (5), bulk (0)"""
        out = np.zeros((10, self.n))
        self._chk(A.lib().vh_get_conserved(self.h, A.ptr(out)))
        return out

    def get_ns_pi(self) -> np.ndarray:
        """Navier-Stokes 2 eta sigma^{mu nu} (10, n: tt tx ty te xx xy xe yy ye ee)"""
        out = np.zeros((10, self.n))
        self._chk(A.lib().vh_get_ns_pi(self.h, A.ptr(out)))
        return out

    def init_tmunu(self, tau: float, tmunu10: np.ndarray) -> int:
        """state from T^{mu nu} (10, n) by Landau matching; returns the cells
        without a timelike eigenpair (raises when there are any)"""
        t = np.ascontiguousarray(tmunu10, dtype=np.float64).reshape(10, self.n)
        nf = ctypes.c_longlong()
        self._chk(A.lib().vh_init_tmunu(self.h, tau, A.ptr(t), ctypes.byref(nf)))
        return nf.value

    def init_prevu_tmunu(self, tau_prev: float, tmunu10: np.ndarray) -> int:
        """prevu from T^{mu nu} (10, n) at tau_prev by Landau matching"""
        t = np.ascontiguousarray(tmunu10, dtype=np.float64).reshape(10, self.n)
        nf = ctypes.c_longlong()
        self._chk(A.lib().vh_init_prevu_tmunu(self.h, tau_prev, A.ptr(t), ctypes.byref(nf)))
        return nf.value

    def init_profile(self, tau, e, ux, uy, ueta=None, prevu=None, pi_mode=A.PI_ZERO, pi5=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        self._chk(A.lib().vh_init_profile(self.h, tau, A.ptr(c(e)), A.ptr(c(ux)), A.ptr(c(uy)), A.ptr(c(ueta)),
                                          A.ptr(c(prevu)), pi_mode, A.ptr(c(pi5))))

    # ---- evolution
    def step(self, nsteps: int = 1):
        self._chk(A.lib().vh_step(self.h, nsteps))

    @property
    def tau(self) -> float:
        t = ctypes.c_double()
        self._chk(A.lib().vh_get_time(self.h, ctypes.byref(t)))
        return t.value

    def time_kernels(self, nsteps: int) -> np.ndarray:
        out = np.zeros(5)
        self._chk(A.lib().vh_time_kernels(self.h, nsteps, A.ptr(out)))
        return out

    def last_iterations(self) -> int:
        v = ctypes.c_longlong()
        self._chk(A.lib().vh_last_iterations(self.h, ctypes.byref(v)))
        return v.value

    def sweep_uses_tma(self) -> bool:
        """True when the flux sweeps stage their tiles by TMA box copies"""
        v = ctypes.c_int()
        self._chk(A.lib().vh_sweep_uses_tma(self.h, ctypes.byref(v)))
        return bool(v.value)

    # ---- diagnostics
    def max_temperature(self) -> float:
        t = ctypes.c_double()
        self._chk(A.lib().vh_max_temperature(self.h, ctypes.byref(t)))
        return t.value

    def conservation_sums(self) -> np.ndarray:
        out = np.zeros(4)
        self._chk(A.lib().vh_conservation_sums(self.h, A.ptr(out)))
        return out

    def cfl(self):
        a, d = ctypes.c_double(), ctypes.c_double()
        self._chk(A.lib().vh_cfl(self.h, ctypes.byref(a), ctypes.byref(d)))
        return a.value, d.value

    def freezeout_step(self, t_fo: float):
        """the surface T = t_fo swept since the last call, on the GPU
        (vh_freezeout_step): a (count, 9) float64 CUDA tensor on
        boost-invariant grids, (count, 12) in 3+1D; empty on the first call
        after the state is set"""
        import torch
        width = 9 if self.cfg.boost_invariant else 12
        cnt = ctypes.c_longlong()
        rc = A.lib().vh_freezeout_step(self.h, t_fo, None, 0, ctypes.byref(cnt))  # counts (keeps the slice)
        if rc == A.OK:
            return torch.zeros((0, width), dtype=torch.float64, device="cuda")
        if rc != A.E_ARG or cnt.value <= 0:
            self._chk(rc)
        out = torch.zeros((cnt.value, width), dtype=torch.float64, device="cuda")
        self._chk(A.lib().vh_freezeout_step(self.h, t_fo, out.data_ptr(), cnt.value, ctypes.byref(cnt)))
        return out[:cnt.value]

    def write(self, path: str, layout: int = A.WRITE_XY, every: int = 1):
        self._chk(A.lib().vh_write(self.h, path.encode(), layout, every))

    def save_checkpoint(self, path: str):
        self._chk(A.lib().vh_save_checkpoint(self.h, path.encode()))

    def load_checkpoint(self, path: str) -> float:
        """restores the state and time saved by save_checkpoint; returns tau"""
        t = ctypes.c_double()
        self._chk(A.lib().vh_load_checkpoint(self.h, path.encode(), ctypes.byref(t)))
        return t.value

    # ---- observable and its adjoint
    def eps_p(self) -> float:
        v = ctypes.c_double()
        self._chk(A.lib().vh_eps_p(self.h, ctypes.byref(v)))
        return v.value

    def adjoint_eps_p(self, nsteps: int, checkpoint_every: int = 25, want_state: bool = True):
        """eps_p after nsteps steps and its gradients: (eps_p, d/d state (18, n)
        or None, d/d e of init_profile (n,), d/d (etas0, etas1)).  The handle
        is left at the final state."""
        v = ctypes.c_double()
        gs = np.zeros((A.NFIELDS, self.n)) if want_state else None
        ge = np.zeros(self.n)
        gc = np.zeros(2)
        self._chk(A.lib().vh_adjoint_eps_p(self.h, nsteps, checkpoint_every, ctypes.byref(v), A.ptr(gs), A.ptr(ge),
                                           A.ptr(gc)))
        return v.value, gs, ge, gc

    def adjoint_phase_times(self) -> np.ndarray:
        """device ms of the last adjoint: forward, recompute, reverse, rest"""
        out = np.zeros(4)
        self._chk(A.lib().vh_adjoint_phase_times(self.h, A.ptr(out)))
        return out

    def debug_stage_terms(self):
        res = np.zeros((9, self.n)); src = np.zeros((9, self.n)); du = np.zeros((16, self.n))
        self._chk(A.lib().vh_debug_stage_terms(self.h, A.ptr(res), A.ptr(src), A.ptr(du)))
        return res, src, du


# ------------------------------------------------------------ generators

def eos_table_synthetic(n=2000, emin=1e-3, emax=500.0, a=A_QGP, hbarc=HBARC) -> np.ndarray:
    t = np.zeros((4, n))
    A.check(A.lib().vh_eos_table_synthetic(n, emin, emax, a, hbarc, A.ptr(t[0]), A.ptr(t[1]), A.ptr(t[2]),
                                           A.ptr(t[3])))
    return t


def landau_match(tmunu10: np.ndarray, tau: float, cartesian: bool = False):
    """e (n,), u (4, n) and the failure count of the Landau matching of
    T^{mu nu} (10, n) on the GPU (vh_landau_match)"""
    t = np.ascontiguousarray(tmunu10, dtype=np.float64)
    n = t.shape[1]
    e, u = np.zeros(n), np.zeros((4, n))
    nf = ctypes.c_longlong()
    A.check(A.lib().vh_landau_match(A.ptr(t), n, tau, int(cartesian), A.ptr(e), A.ptr(u), ctypes.byref(nf)))
    return e, u, nf.value


def freezeout_2d(nx, ny, dx, dy, tau0, tau1, T0, T1, u0, u1, t_fo):
    """the isothermal surface T = t_fo between two time slices of a
    boost-invariant run: (count, 9) rows of centroid (tau, x, y), dSigma_mu
    per unit rapidity (tau, x, y) and u^tau, u^x, u^y"""
    c = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    T0, T1, u0, u1 = c(T0), c(T1), c(np.asarray(u0)[:3]), c(np.asarray(u1)[:3])
    cnt = ctypes.c_longlong()
    args = (nx, ny, dx, dy, tau0, tau1, A.ptr(T0), A.ptr(T1), A.ptr(u0), A.ptr(u1), t_fo)
    A.lib().vh_freezeout_2d(*args, None, 0, ctypes.byref(cnt))  # counts the elements
    out = np.zeros((max(cnt.value, 1), 9))
    A.check(A.lib().vh_freezeout_2d(*args, A.ptr(out), cnt.value, ctypes.byref(cnt)))
    return out[:cnt.value]


def cooper_frye_2d(elements, t_fo, mass, degeneracy, pt, phi):
    """Boltzmann E dN/d^3p at mid-rapidity (len(pt), len(phi)) from the
    elements of freezeout_2d"""
    el = np.ascontiguousarray(elements, dtype=np.float64).reshape(-1, 9)
    pt = np.ascontiguousarray(pt, dtype=np.float64).reshape(-1)
    phi = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
    out = np.zeros((pt.size, phi.size))
    A.check(A.lib().vh_cooper_frye_2d(A.ptr(el), el.shape[0], t_fo, mass, degeneracy, A.ptr(pt), pt.size, A.ptr(phi),
                                      phi.size, A.ptr(out)))
    return out


def cooper_frye_3d(elements, t_fo, mass, degeneracy, y, pt, phi):
    """Boltzmann E dN/d^3p at rapidity y (len(pt), len(phi)) from the
    elements of freezeout_3d"""
    el = np.ascontiguousarray(elements, dtype=np.float64).reshape(-1, 12)
    pt = np.ascontiguousarray(pt, dtype=np.float64).reshape(-1)
    phi = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
    out = np.zeros((pt.size, phi.size))
    A.check(A.lib().vh_cooper_frye_3d(A.ptr(el), el.shape[0], t_fo, mass, degeneracy, y, A.ptr(pt), pt.size,
                                      A.ptr(phi), phi.size, A.ptr(out)))
    return out


def freezeout_3d(nx, ny, nz, dx, dy, dz, tau0, tau1, T0, T1, u0, u1, t_fo):
    """the isothermal surface T = t_fo between two time slices of a 3+1D
    run: (count, 12) rows of centroid (tau, x, y, eta), dSigma_mu (tau, x,
    y, eta) and u^mu"""
    c = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    T0, T1, u0, u1 = c(T0), c(T1), c(np.asarray(u0)[:4]), c(np.asarray(u1)[:4])
    cnt = ctypes.c_longlong()
    args = (nx, ny, nz, dx, dy, dz, tau0, tau1, A.ptr(T0), A.ptr(T1), A.ptr(u0), A.ptr(u1), t_fo)
    A.lib().vh_freezeout_3d(*args, None, 0, ctypes.byref(cnt))  # counts the elements
    out = np.zeros((max(cnt.value, 1), 12))
    A.check(A.lib().vh_freezeout_3d(*args, A.ptr(out), cnt.value, ctypes.byref(cnt)))
    return out[:cnt.value]


def flow_coefficients(spectrum, phi, orders=(1, 2, 3, 4)):
    """anisotropic flow of spectra (len(pt), len(phi)) on a uniform azimuth
    grid over [0, 2 pi): v_n(p_T) = |sum_b S e^{i n phi_b}| / sum_b S and the
    event-plane angle Psi_n = arg(sum_b S e^{i n phi_b}) / n, for each order
    (exact for harmonics below len(phi) / 2); returns v, psi of shape
    (len(orders), len(pt))"""
    S = np.asarray(spectrum, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64).reshape(-1)
    if S.ndim != 2 or S.shape[1] != phi.size:
        raise ValueError("spectrum must be (len(pt), len(phi))")
    step = 2 * np.pi / phi.size
    if not np.allclose(np.diff(phi), step, rtol=0, atol=1e-12 * step):
        raise ValueError("phi must be a uniform grid over [0, 2 pi)")
    q = np.array([(S * np.exp(1j * n * phi)[None, :]).sum(axis=1) for n in orders]) / S.sum(axis=1)[None, :]
    return np.abs(q), np.angle(q) / np.asarray(orders, dtype=np.float64)[:, None]


def _cuda_f64(t, rows, n):
    """rows x n float64 values of a CUDA tensor, contiguous (a copy only when
    needed); rows = 0 for a flat array of n"""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError("expected a CUDA tensor")
    t = t.to(torch.float64).reshape(-1, n) if rows else t.to(torch.float64).reshape(-1)
    if rows:
        if t.shape[0] < rows:
            raise ValueError(f"expected at least {rows} rows of {n}")
        t = t[:rows]
    elif t.numel() != n:
        raise ValueError(f"expected {n} values")
    return t.contiguous()


def _stream(stream):
    import torch
    return torch.cuda.current_stream().cuda_stream if stream is None else stream


def _surface_device(fn, width, rows, geo, n, T0, T1, u0, u1, t_fo, stream):
    import torch
    ts = [_cuda_f64(T0, 0, n), _cuda_f64(T1, 0, n), _cuda_f64(u0, rows, n), _cuda_f64(u1, rows, n)]
    args = (*geo, *[t.data_ptr() for t in ts], t_fo)
    cnt = ctypes.c_longlong()
    st = _stream(stream)
    rc = fn(*args, None, 0, ctypes.byref(cnt), st)  # counts the elements
    if rc not in (A.OK, A.E_ARG) or cnt.value < 0:
        A.check(rc)
    out = torch.zeros((max(cnt.value, 1), width), dtype=torch.float64, device=ts[0].device)
    A.check(fn(*args, out.data_ptr(), cnt.value, ctypes.byref(cnt), st))
    return out[:cnt.value]


def freezeout_2d_device(nx, ny, dx, dy, tau0, tau1, T0, T1, u0, u1, t_fo, stream=None):
    """freezeout_2d on the GPU (vh_freezeout_2d_device): T0, T1 and u0, u1
    (u^tau, u^x, u^y rows) as CUDA tensors on the ghost-inclusive grid; a
    (count, 9) float64 CUDA tensor in freezeout_2d's element order"""
    n = (nx + 6) * (ny + 6)
    return _surface_device(A.lib().vh_freezeout_2d_device, 9, 3, (nx, ny, dx, dy, tau0, tau1), n, T0, T1, u0, u1,
                           t_fo, stream)


def freezeout_3d_device(nx, ny, nz, dx, dy, dz, tau0, tau1, T0, T1, u0, u1, t_fo, stream=None):
    """freezeout_3d on the GPU (vh_freezeout_3d_device): a (count, 12)
    float64 CUDA tensor in freezeout_3d's element order"""
    n = (nx + 6) * (ny + 6) * (nz + 6)
    return _surface_device(A.lib().vh_freezeout_3d_device, 12, 4, (nx, ny, nz, dx, dy, dz, tau0, tau1), n, T0, T1,
                           u0, u1, t_fo, stream)


def cooper_frye_2d_device(elements, t_fo, mass, degeneracy, pt, phi, stream=None):
    """cooper_frye_2d from elements in a CUDA tensor (count, 9), summed on
    the GPU (vh_cooper_frye_2d_device); a (len(pt), len(phi)) array"""
    el = _cuda_f64(elements, 0, elements.numel())
    pt = np.ascontiguousarray(pt, dtype=np.float64).reshape(-1)
    phi = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
    out = np.zeros((pt.size, phi.size))
    A.check(A.lib().vh_cooper_frye_2d_device(el.data_ptr(), el.numel() // 9, t_fo, mass, degeneracy, A.ptr(pt),
                                             pt.size, A.ptr(phi), phi.size, A.ptr(out), _stream(stream)))
    return out


def cooper_frye_3d_device(elements, t_fo, mass, degeneracy, y, pt, phi, stream=None):
    """cooper_frye_3d from elements in a CUDA tensor (count, 12), summed on
    the GPU (vh_cooper_frye_3d_device); a (len(pt), len(phi)) array"""
    el = _cuda_f64(elements, 0, elements.numel())
    pt = np.ascontiguousarray(pt, dtype=np.float64).reshape(-1)
    phi = np.ascontiguousarray(phi, dtype=np.float64).reshape(-1)
    out = np.zeros((pt.size, phi.size))
    A.check(A.lib().vh_cooper_frye_3d_device(el.data_ptr(), el.numel() // 12, t_fo, mass, degeneracy, y, A.ptr(pt),
                                             pt.size, A.ptr(phi), phi.size, A.ptr(out), _stream(stream)))
    return out


def profile_gubser_cold(nx, ny, dx, dy, q=1.0, tau0=1.0, dtau=0.01, b=1.21, a=A_QGP):
    """the cold-plasma viscous Gubser flow at tau0: e, u^x, u^y, pi5 and prevu
    (at tau0 - dtau) on the 2+1D ghost-inclusive grid"""
    n = (nx + 6) * (ny + 6)
    e, ux, uy, pi5, pu = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros((5, n)), np.zeros((4, n))
    A.check(A.lib().vh_profile_gubser_cold(nx, ny, dx, dy, q, tau0, dtau, b, a, A.ptr(e), A.ptr(ux), A.ptr(uy),
                                           A.ptr(pi5), A.ptr(pu)))
    return e, ux, uy, pi5, pu


def profile_gubser_is(nx, ny, dx, dy, q=1.0, tau0=1.0, dtau=0.01, t0_gev=0.6, p0=0.0, etas=0.2, a=A_QGP,
                      hbarc=HBARC):
    """the Israel-Stewart Gubser flow at tau0 (T = t0_gev and shear ratio
    tau^2 pi^{eta eta}/(e+P) = p0 at the grid centre): e, u^x, u^y, pi5 and
    prevu (at tau0 - dtau) on the 2+1D ghost-inclusive grid"""
    n = (nx + 6) * (ny + 6)
    e, ux, uy, pi5, pu = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros((5, n)), np.zeros((4, n))
    A.check(A.lib().vh_profile_gubser_is(nx, ny, dx, dy, q, tau0, dtau, t0_gev, p0, etas, a, hbarc, A.ptr(e),
                                         A.ptr(ux), A.ptr(uy), A.ptr(pi5), A.ptr(pu)))
    return e, ux, uy, pi5, pu


def profile_cgc(nx, ny, nz=1, boost_invariant=True, dx=0.1, dy=0.1, dz=0.1, tau=0.1, e_peak=1.0, x_pos=3.0,
                mass_number=197.0, ws_a=0.546, thickness_scale=12.2546, eta_flat=4.0, delta=100.0) -> np.ndarray:
    """the optical-Glauber CGC T^{mu nu} (10, n) of the reference's Glasma
    initialisation on the ghost-inclusive grid (host code)"""
    gz = 1 if boost_invariant else nz + 6
    out = np.zeros((10, (nx + 6) * (ny + 6) * gz))
    A.check(A.lib().vh_profile_cgc(nx, ny, nz, int(boost_invariant), dx, dy, dz, tau, x_pos, mass_number, ws_a,
                                   thickness_scale, e_peak, eta_flat, delta, A.ptr(out)))
    return out


def read_ideal_profile(eps_path: str, vx_path: str, vy_path: str, nx: int, ny: int):
    """e, u^x, u^y on the ghost-inclusive (nx+6)x(ny+6) grid from the ideal
    driver's ASCII files, and the floor's min (vh_read_ideal_profile)."""
    g = (nx + 6) * (ny + 6)
    e, ux, uy = np.zeros(g), np.zeros(g), np.zeros(g)
    mn = ctypes.c_double()
    A.check(A.lib().vh_read_ideal_profile(eps_path.encode(), vx_path.encode(), vy_path.encode(), nx, ny, A.ptr(e),
                                          A.ptr(ux), A.ptr(uy), ctypes.byref(mn)))
    return e, ux, uy, mn.value


def profile_gubser(nx, ny, dx, dy, q=1.0, tau0=1.0, dtau=0.01, t0_gev=0.6, a=A_QGP, hbarc=HBARC):
    gx, gy = nx + 6, ny + 6
    e = np.zeros(gx * gy); ux = np.zeros_like(e); uy = np.zeros_like(e); pu = np.zeros(4 * gx * gy)
    A.check(A.lib().vh_profile_gubser(nx, ny, dx, dy, q, tau0, dtau, t0_gev, a, hbarc, A.ptr(e), A.ptr(ux),
                                      A.ptr(uy), A.ptr(pu)))
    return e, ux, uy, pu


def profile_glauber(nx, ny, nz=1, boost_invariant=True, dx=0.1, dy=0.1, dz=0.25, A_nuc=208, R=6.62, aws=0.546,
                    dmin=0.4, b=7.0, sigma_nn=6.4, w=0.5, epeak_gev=40.0, eta_flat=1.5, eta_sigma=1.3,
                    efloor_gev=0.04, hbarc=HBARC, seed=0):
    gz = 1 if boost_invariant else nz + 6
    e = np.zeros((nx + 6) * (ny + 6) * gz)
    npart = ctypes.c_int()
    A.check(A.lib().vh_profile_glauber(nx, ny, nz, int(boost_invariant), dx, dy, dz, A_nuc, R, aws, dmin, b,
                                       sigma_nn, w, epeak_gev, eta_flat, eta_sigma, efloor_gev, hbarc, seed, A.ptr(e),
                                       ctypes.byref(npart)))
    return e, npart.value
