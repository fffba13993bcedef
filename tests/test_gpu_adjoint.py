"""The discrete adjoint through the C ABI (vh_adjoint_eps_p) against central
finite differences of the forward step, in FP64 and in the mixed mode.

The observable is the momentum anisotropy eps_p at the final time of a
boost-invariant MC-Glauber event (b = 7 fm, seed 0) with eta/s(T) = c0 +
c1 max(T - 0.154 GeV, 0), c0 = 0.08, c1 = 1.0 GeV^-1.  Energy-density
directions are unit vectors v over the interior cells (e0 -> e0 + h v, e0
in fm^-4); c0 and c1 are perturbed relatively (c -> c (1 + h)); h = 1e-6.

The 330-step event (tau 0.6 -> 7.2 fm/c) is sensitive to its initial state:
a relative perturbation of 1e-7 changes the FP64 gradient field by ~17 %
(measured), growing exponentially after tau ~ 2.6 fm/c.  So the strict 1e-4
finite-difference bar is applied at 100 steps, the full event is held to its
median, and the mixed mode is compared with FP64 where the trajectories have
not yet separated.  The gradient is wrapped in a torch.autograd.Function
here, in the tests only.
"""
import numpy as np
import pytest
import torch

from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Hydro

pytestmark = pytest.mark.gpu

H = 1e-6


class Event:
    """One Glauber event evolved nsteps steps from tau0 = 0.6 fm/c."""

    def __init__(self, side, nsteps, precision=A.PREC_FP64, c0=0.08, c1=1.0, floor=C.ADJOINT_FLOOR_GEV):
        self.side, self.nsteps, self.precision = side, nsteps, precision
        self.c = np.array([c0, c1])
        self.inp = C.glauber_inputs(self.cfg(self.c), b=7.0, seed=0, efloor_gev=floor)
        self.e0 = self.inp["e"].copy()
        g = side + 6
        m = np.zeros((g, g), dtype=bool)
        m[3:3 + side, 3:3 + side] = True
        self.interior = m.reshape(-1)

    def cfg(self, c, precision=None):
        return C.adjoint_config(self.side, self.precision if precision is None else precision, float(c[0]),
                                float(c[1]))

    def hydro(self, e0, c, precision=None):
        h = Hydro(self.cfg(c, precision))
        i = self.inp
        h.init_profile(i["tau"], e0, i["ux"], i["uy"], i["ueta"], i["prevu"], i["pi_mode"])
        return h

    def eps(self, e0=None, c=None, precision=None):
        with self.hydro(self.e0 if e0 is None else e0, self.c if c is None else c, precision) as h:
            h.step(self.nsteps)
            return h.eps_p()

    def adjoint(self, e0=None, c=None, every=25, precision=None, want_state=False):
        with self.hydro(self.e0 if e0 is None else e0, self.c if c is None else c, precision) as h:
            out = h.adjoint_eps_p(self.nsteps, every, want_state=want_state)
            assert abs(h.tau - (0.6 + self.nsteps * 0.02)) < 1e-9
            return out

    def direction(self, v):
        d = np.zeros_like(self.e0)
        d[self.interior] = v
        return d

    def fd_e(self, v, h=None):
        h = H if h is None else h
        d = self.direction(v)
        return (self.eps(self.e0 + h * d) - self.eps(self.e0 - h * d)) / (2 * h)

    def fd_c(self, k, h=None):
        h = H if h is None else h
        cp = self.c.copy(); cm = self.c.copy()
        cp[k] *= 1 + h; cm[k] *= 1 - h
        return (self.eps(c=cp) - self.eps(c=cm)) / (2 * h * self.c[k])


def unit_directions(ev, count, seed=1234):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        v = rng.normal(size=int(ev.interior.sum()))
        out.append(v / np.linalg.norm(v))
    return out


def fd_errors(ev, ge, gc, ndir):
    errs = []
    for v in unit_directions(ev, ndir):
        fd = ev.fd_e(v)
        errs.append(abs(float(np.dot(ge, ev.direction(v))) - fd) / abs(fd))
    cerr = [abs(gc[k] - ev.fd_c(k)) / abs(ev.fd_c(k)) for k in range(2)]
    return np.array(errs), np.array(cerr)


class EpsP(torch.autograd.Function):
    """eps_p(e0 on the interior, (c0, c1)) with the adjoint as its backward."""

    @staticmethod
    def forward(ctx, e_int, c, ev):
        e0 = ev.e0.copy()
        e0[ev.interior] = e_int.detach().cpu().numpy()
        eps, _, ge, gc = ev.adjoint(e0, c.detach().cpu().numpy())
        ctx.save_for_backward(torch.from_numpy(ge[ev.interior].copy()), torch.from_numpy(gc.copy()))
        return torch.tensor(eps, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        ge, gc = ctx.saved_tensors
        return g * ge, g * gc, None


def test_finite_differences_converge_to_the_adjoint():
    """40 steps of a 24x24 event: central differences with h = 1e-4 and 1e-5
    agree with the adjoint to 1e-6; at h = 1e-6 (4e-8 per cell) the
    forward's rounding shows in the difference, at the 1e-6 level"""
    ev = Event(side=24, nsteps=40)
    eps, _, ge, gc = ev.adjoint(every=7)
    assert abs(eps - ev.eps()) <= 1e-14 * abs(eps)
    for v in unit_directions(ev, 3):
        ad = float(np.dot(ge, ev.direction(v)))
        err = [abs(ad - ev.fd_e(v, h)) / abs(ad) for h in (1e-4, 1e-5, 1e-6)]
        assert err[0] <= 1e-6 and err[1] <= 1e-6 and err[2] <= 1e-5, err
    for k in range(2):
        assert abs(gc[k] - ev.fd_c(k)) <= 1e-6 * abs(gc[k])


def test_per_cell_state_gradient():
    """every state field of every cell, one step at a time: 10x10 smooth
    viscous state, conformal EOS (no table nodes), 4 steps"""
    from helpers import oracle_config, smooth_inputs
    from pyoracle import Oracle
    from viral_b200.hydro import Config
    cfg = Config(nx=10, ny=10, eos_kind=A.EOS_CONFORMAL, etas0=0.2, etas1=0.0, taupi_kind=A.TAUPI_15_ETA_OVER_P)
    s0 = smooth_inputs(cfg, cfg.tau0, seed=3)
    s0[4] = 0; s0[8] = 0; s0[9] = 0; s0[17] = 0  # boost invariance: u^eta = pi^{x eta} = pi^{y eta} = 0
    s0[1] = np.sqrt(1 + s0[2] ** 2 + s0[3] ** 2)
    s0[14] = np.sqrt(1 + s0[15] ** 2 + s0[16] ** 2)
    O = Oracle(oracle_config(cfg))
    O.set_state(s0)
    O.fill_tmunu(cfg.tau0)
    s0 = O.get_state()
    nsteps = 4
    with Hydro(cfg) as h:
        h.set_state(s0, cfg.tau0)
        _, gs, _, _ = h.adjoint_eps_p(nsteps, 3)

        def f(s):
            h.set_state(s, cfg.tau0)
            h.step(nsteps)
            return h.eps_p()

        for fld in (0, 2, 3, 5, 6, 7, 10, 11, 12, 15, 16):
            fd = np.zeros(s0.shape[1])
            dh = 1e-6 * max(np.abs(s0[fld]).max(), 1e-3)
            for c in range(s0.shape[1]):
                sp = s0.copy(); sp[fld, c] += dh
                sm = s0.copy(); sm[fld, c] -= dh
                fd[c] = (f(sp) - f(sm)) / (2 * dh)
            assert np.abs(gs[fld] - fd).max() <= 1e-5 * np.abs(fd).max(), fld


def test_checkpoint_interval_does_not_change_the_gradient():
    ev = Event(side=20, nsteps=30)
    ref = ev.adjoint(every=30, want_state=True)
    for every in (1, 7):
        got = ev.adjoint(every=every, want_state=True)
        assert got[0] == ref[0]
        for q in (1, 2, 3):
            assert np.array_equal(got[q], ref[q])


def test_glauber_128_fp64_to_tau_2_6():
    """the 128x128 event, 100 steps: every direction within 1e-4"""
    ev = Event(side=128, nsteps=100)
    eps, _, ge, gc = ev.adjoint(every=25)
    errs, cerr = fd_errors(ev, ge, gc, 16)
    print("128^2 FP64 100 steps: eps_p %.8f; e0 directions max %.2e median %.2e; (c0, c1) %s" % (
        eps, errs.max(), np.median(errs), cerr))
    assert errs.max() <= 1e-4 and cerr.max() <= 1e-4


def test_glauber_128_fp64_to_tau_7_2():
    """the full 330-step event, checkpoints every 25 steps, 16 directions"""
    ev = Event(side=128, nsteps=C.ADJOINT_STEPS)
    eps, _, ge, gc = ev.adjoint(every=25)
    errs, cerr = fd_errors(ev, ge, gc, 16)
    print("128^2 FP64 330 steps: eps_p %.8f; e0 directions %s; (c0, c1) %s" % (
        eps, ["%.1e" % x for x in errs], cerr))
    assert np.median(errs) <= 1e-4 and np.sum(errs <= 1e-4) >= 12 and errs.max() <= 1e-2
    assert cerr.max() <= 1e-4


def test_glauber_128_mixed_against_fp64():
    """the mixed adjoint (FP32, implicit-function solve in FP64) against the
    FP64 adjoint and the FP64 forward's finite differences, 100 steps; the
    agreement is bounded by the FP32 trajectory, which the FP64 gradient is
    sensitive to (a 1e-7 perturbation of e0 moves its field by 1e-3)"""
    ev = Event(side=128, nsteps=100)
    eps64, _, ge64, gc64 = ev.adjoint(every=25)
    eps32, _, ge32, gc32 = ev.adjoint(every=25, precision=A.PREC_MIXED)
    m = ev.interior
    w = ev.e0[m]
    field = np.linalg.norm((ge32 - ge64)[m] * w) / np.linalg.norm(ge64[m] * w)
    cdiff = np.abs(gc32 - gc64) / np.abs(gc64)
    errs = []
    errs64 = []
    for v in unit_directions(ev, 16):
        fd = ev.fd_e(v)
        errs.append(abs(float(np.dot(ge32, ev.direction(v))) - fd) / abs(fd))
        errs64.append(abs(float(np.dot(ge64, ev.direction(v))) - fd) / abs(fd))
    print("128^2 mixed 100 steps: field %.2e, (c0, c1) %s, vs FP64 FD max %.2e median %.2e (FP64 adjoint: max %.2e)"
          % (field, cdiff, max(errs), float(np.median(errs)), max(errs64)))
    assert abs(eps32 - eps64) <= 1e-5 * abs(eps64)
    assert field <= 5e-3 and cdiff.max() <= 1e-4 and max(errs) <= 5e-2


def test_autograd_function_wraps_the_adjoint():
    ev = Event(side=20, nsteps=20)
    e_int = torch.tensor(ev.e0[ev.interior], dtype=torch.float64, requires_grad=True)
    c = torch.tensor(ev.c, dtype=torch.float64, requires_grad=True)
    y = EpsP.apply(e_int, c, ev)
    y.backward()
    v = unit_directions(ev, 1, seed=99)[0]
    fd = ev.fd_e(v)
    assert abs(float(torch.dot(e_int.grad, torch.from_numpy(v))) - fd) <= 1e-5 * abs(fd)
    assert abs(float(c.grad[1]) - ev.fd_c(1)) <= 1e-5 * abs(ev.fd_c(1))


def test_unsupported_configurations_are_refused():
    """minmod reconstruction and Cartesian coordinates have no adjoint (3+1D
    Milne grids do: tests/test_gpu_adjoint3.py)"""
    for cfg in (C.glauber_config(nx=16, ny=16, nz=8, boost_invariant=False, recon=A.RECON_MINMOD),
                C.glauber_config(nx=16, ny=16, boost_invariant=True, recon=A.RECON_MINMOD)):
        with Hydro(cfg) as h:
            inp = C.glauber_inputs(cfg)
            h.init_profile(inp["tau"], inp["e"], inp["ux"], inp["uy"], inp["ueta"], None, inp["pi_mode"])
            with pytest.raises(A.VhError) as ex:
                h.adjoint_eps_p(2, 1)
            assert ex.value.code == A.E_UNSUPPORTED
    cart = C.cart_bjorken_config()
    with Hydro(cart) as h:
        n = h.n
        s = np.zeros((A.NFIELDS, n))
        s[0] = 1.0; s[1] = 1.0; s[14] = 1.0
        h.set_state(s, cart.tau0)
        with pytest.raises(A.VhError) as ex:
            h.adjoint_eps_p(2, 1)
        assert ex.value.code == A.E_UNSUPPORTED
