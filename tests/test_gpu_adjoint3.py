"""The 3+1D discrete adjoint through the C ABI (vh_adjoint_eps_p on a grid
that is not boost invariant) against central finite differences of the
forward step.  The observable is eps_p over every interior cell (all eta
slices) at the final time.

* every one of the 18 state fields, cell by cell (a sample of the cells per
  field, ghosts included), on a small smooth viscous state with u^eta,
  pi^{x eta}, pi^{y eta} and T^{tau eta} all nonzero;
* a 3+1D MC-Glauber event with the table EOS and eta/s(T) = c0 + c1 max(T -
  0.154 GeV, 0): unit directions of the initial energy density and (c0, c1);
* the checkpoint interval does not change the gradient (bitwise);
* the mixed mode against FP64 on the same event.
"""
import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Config, Hydro

pytestmark = pytest.mark.gpu


def _smooth_3d(cfg, seed):
    from helpers import oracle_config, smooth_inputs
    from pyoracle import Oracle
    s0 = smooth_inputs(cfg, cfg.tau0, seed=seed)
    O = Oracle(oracle_config(cfg))
    O.set_state(s0)
    O.fill_tmunu(cfg.tau0)
    return O.get_state()


def test_3d_per_cell_state_gradient():
    """8x7x6 smooth viscous state, conformal EOS, 3 steps: every field, 30
    cells per field (interior and ghost), within 1e-5 of the largest FD
    derivative of that field.  The differences are Richardson-extrapolated
    from steps of 4e-6 and 2e-6 of the field's scale: plain central
    differences leave an h^2 error of 2.5e-6 in e at 1e-6 (2.6e-4 at 1e-5),
    while rounding of eps_p reaches 1.2e-5 of the small pi^{y eta}
    differences at 1e-6 (measured)"""
    cfg = Config(nx=8, ny=7, nz=6, boost_invariant=False, dx=0.15, dy=0.15, dz=0.1, eos_kind=A.EOS_CONFORMAL,
                 etas0=0.2, etas1=0.0, taupi_kind=A.TAUPI_15_ETA_OVER_P)
    s0 = _smooth_3d(cfg, seed=5)
    nsteps = 3
    rng = np.random.default_rng(17)
    with Hydro(cfg) as h:
        h.set_state(s0, cfg.tau0)
        eps, gs, _, _ = h.adjoint_eps_p(nsteps, 2)

        def f(s):
            h.set_state(s, cfg.tau0)
            h.step(nsteps)
            return h.eps_p()

        assert abs(f(s0) - eps) <= 1e-14 * abs(eps)
        def central(fld, c, dh):
            sp = s0.copy(); sp[fld, c] += dh
            sm = s0.copy(); sm[fld, c] -= dh
            return (f(sp) - f(sm)) / (2 * dh)

        worst = {}
        for fld in range(18):
            cells = rng.choice(s0.shape[1], size=30, replace=False)
            dh = 4e-6 * max(np.abs(s0[fld]).max(), 1e-3)
            # Richardson: (4 D(h/2) - D(h)) / 3 cancels the h^2 term
            fd = np.array([(4 * central(fld, c, dh / 2) - central(fld, c, dh)) / 3 for c in cells])
            scale = max(np.abs(fd).max(), np.abs(gs[fld]).max(), 1e-12)
            worst[fld] = float(np.abs(gs[fld, cells] - fd).max() / scale)
        print("3+1D per-cell gradient, worst relative error per field:", {k: "%.1e" % v for k, v in worst.items()})
        assert max(worst.values()) <= 1e-5, worst


class Event3:
    """A 3+1D Glauber event evolved nsteps steps from tau0 = 0.6 fm/c."""

    def __init__(self, nx, ny, nz, nsteps, precision=A.PREC_FP64, c0=0.08, c1=1.0):
        self.dims, self.nsteps, self.precision = (nx, ny, nz), nsteps, precision
        self.c = np.array([c0, c1])
        self.inp = C.glauber_inputs(self.cfg(self.c), b=7.0, seed=3, efloor_gev=C.ADJOINT_FLOOR_GEV)
        self.e0 = self.inp["e"].copy()
        gx, gy, gz = nx + 6, ny + 6, nz + 6
        m = np.zeros((gz, gy, gx), dtype=bool)
        m[3:3 + nz, 3:3 + ny, 3:3 + nx] = True
        self.interior = m.reshape(-1)

    def cfg(self, c, precision=None):
        nx, ny, nz = self.dims
        return C.glauber_config(nx=nx, ny=ny, nz=nz, boost_invariant=False,
                                precision=self.precision if precision is None else precision,
                                etas0=float(c[0]), etas1=float(c[1]))

    def hydro(self, e0, c, precision=None):
        h = Hydro(self.cfg(c, precision))
        i = self.inp
        h.init_profile(i["tau"], e0, i["ux"], i["uy"], i["ueta"], i["prevu"], i["pi_mode"])
        return h

    def eps(self, e0=None, c=None):
        with self.hydro(self.e0 if e0 is None else e0, self.c if c is None else c) as h:
            h.step(self.nsteps)
            return h.eps_p()

    def adjoint(self, every=10, precision=None, want_state=False):
        with self.hydro(self.e0, self.c, precision) as h:
            return h.adjoint_eps_p(self.nsteps, every, want_state=want_state)

    def direction(self, v):
        d = np.zeros_like(self.e0)
        d[self.interior] = v
        return d

    def fd_e(self, v, h=1e-4):
        d = self.direction(v)
        return (self.eps(self.e0 + h * d) - self.eps(self.e0 - h * d)) / (2 * h)

    def fd_c(self, k, h=1e-6):
        cp = self.c.copy(); cm = self.c.copy()
        cp[k] *= 1 + h; cm[k] *= 1 - h
        return (self.eps(c=cp) - self.eps(c=cm)) / (2 * h * self.c[k])


def _directions(ev, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        v = rng.normal(size=int(ev.interior.sum()))
        out.append(v / np.linalg.norm(v))
    return out


def test_3d_glauber_event_against_finite_differences():
    """32x32x12 event, table EOS, eta/s(T) with the kink, 30 steps.  Some
    directional derivatives of eps_p (-6e-4) are as small as 2e-8, so the
    energy-density differences take h = 1e-4 (measured on this event: the
    relative error of the central difference is O(1e-4) at h = 1e-3, from
    truncation, 1e-8..4e-6 at 1e-4, and up to 7e-5 at 1e-6, from rounding)"""
    ev = Event3(32, 32, 12, 30)
    eps, _, ge, gc = ev.adjoint(every=10)
    assert abs(eps - ev.eps()) <= 1e-14 * abs(eps)
    errs = []
    for v in _directions(ev, 6, 7):
        fd = ev.fd_e(v)
        errs.append(abs(float(np.dot(ge, ev.direction(v))) - fd) / abs(fd))
    cerr = [abs(gc[k] - ev.fd_c(k)) / abs(ev.fd_c(k)) for k in range(2)]
    print("3+1D 32x32x12, 30 steps: eps_p %.8f; e0 directions %s; (c0, c1) %s" % (
        eps, ["%.1e" % x for x in errs], ["%.1e" % x for x in cerr]))
    assert max(errs) <= 1e-5 and max(cerr) <= 1e-5


def test_3d_checkpoint_interval_does_not_change_the_gradient():
    ev = Event3(20, 18, 10, 12)
    ref = ev.adjoint(every=12, want_state=True)
    for every in (1, 5):
        got = ev.adjoint(every=every, want_state=True)
        assert got[0] == ref[0]
        for q in (1, 2, 3):
            assert np.array_equal(got[q], ref[q])


def test_3d_mixed_against_fp64():
    ev = Event3(32, 32, 12, 30)
    eps64, _, ge64, gc64 = ev.adjoint(every=10)
    eps32, _, ge32, gc32 = ev.adjoint(every=10, precision=A.PREC_MIXED)
    m = ev.interior
    w = ev.e0[m]
    field = np.linalg.norm((ge32 - ge64)[m] * w) / np.linalg.norm(ge64[m] * w)
    cdiff = np.abs(gc32 - gc64) / np.abs(gc64)
    print("3+1D mixed vs FP64: eps_p %.2e, field %.2e, (c0, c1) %s" % (
        abs(eps32 - eps64) / abs(eps64), field, cdiff))
    assert abs(eps32 - eps64) <= 1e-5 * abs(eps64)
    assert field <= 1e-2 and cdiff.max() <= 1e-3
