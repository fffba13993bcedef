"""The batched ensemble (one persistent kernel over a packed event table)
against the single-event step through the C ABI.

Each batched event must evolve exactly as the same event stepped alone
(same device arithmetic, only the work distribution differs), for every
compiled variant of the persistent kernel, stop at the same step under the
freeze-out rule that the single-event loop applies after every step, and
fail alone without disturbing the others.
"""
import numpy as np
import pytest

from conftest import rel_err
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.batch import EVENT_FAILED, EVENT_FROZEN, EVENT_RUNNING, EVENT_TAUMAX, Batch
from viral_b200.hydro import Hydro

pytestmark = pytest.mark.gpu

SIDES = [24, 33, 41, 27, 58, 30]
BIMP = [2.0, 5.0, 8.0, 3.0, 7.0, 11.0]


def single_event(cfg, side, b, seed, steps):
    c = C.glauber_config(nx=side, ny=side, boost_invariant=True, precision=cfg.precision)
    inp = C.glauber_inputs(c, b=b, seed=seed)
    with C.make_hydro(c, inp) as H:
        H.step(steps)
        return H.get_state()


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_batch_matches_single_events(precision, variant):
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True, precision=precision)
    steps = 12
    with Batch(cfg, SIDES, tau0=cfg.tau0, dtau=cfg.dtau, tau_max=100.0, t_freeze_gev=0.0) as B:
        B.init_glauber(seeds=np.arange(len(SIDES)), bimp=BIMP)
        B.set_tuning(variant, steps_per_launch=4, use_graph=True)
        sec, graph = B.run(steps)
        tau, nst, st = B.events()
        assert np.all(st == EVENT_RUNNING) and np.all(nst == steps)
        assert np.allclose(tau, cfg.tau0 + steps * cfg.dtau)
        # FP64: identical up to rounding; mixed: the same FP32 source compiled
        # into another kernel may fuse multiply-adds differently (ulp level)
        tol = 1e-13 if precision == A.PREC_FP64 else 1e-5
        for ev, (side, b) in enumerate(zip(SIDES, BIMP)):
            ref = single_event(cfg, side, b, ev, steps)
            got = B.event_state(ev)
            for q in range(14):
                assert rel_err(got[q], ref[q]) <= tol, (ev, q)


def test_freeze_out_per_event():
    """Each event stops after the first step whose maximum temperature is
    below the freeze-out value, as the single-event loop decides it."""
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True)
    sides, bimp = [30, 36, 44], [10.0, 6.0, 2.0]
    t_fo = 0.30
    with Batch(cfg, sides, tau0=cfg.tau0, dtau=cfg.dtau, tau_max=3.0, t_freeze_gev=t_fo) as B:
        B.init_glauber(seeds=[5, 6, 7], bimp=bimp)
        B.run(1000)
        tau, nst, st = B.events()
    for ev, (side, b) in enumerate(zip(sides, bimp)):
        c = C.glauber_config(nx=side, ny=side, boost_invariant=True)
        with C.make_hydro(c, C.glauber_inputs(c, b=b, seed=5 + ev)) as H:
            n = 0
            while True:
                H.step(1)
                n += 1
                if H.max_temperature() < t_fo:
                    want = EVENT_FROZEN
                    break
                if H.tau >= 3.0 - 1e-9:
                    want = EVENT_TAUMAX
                    break
        assert st[ev] == want and nst[ev] == n, (ev, st[ev], nst[ev], want, n)


def test_failed_event_does_not_stop_the_others():
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True)
    sides = [24, 24, 24]
    with Batch(cfg, sides, tau0=cfg.tau0, dtau=cfg.dtau, tau_max=100.0, t_freeze_gev=0.0) as B:
        B.init_glauber(seeds=[1, 2, 3], bimp=[4.0, 4.0, 4.0])
        c = C.glauber_config(nx=24, ny=24, boost_invariant=True)
        inp = C.glauber_inputs(c, b=4.0, seed=2)
        bad = inp["e"].copy()
        g = 24 + 6
        bad[15 * g + 15] = -50.0  # an interior cell with negative energy density: its root-find fails
        B.init_event(1, bad, inp["ux"], inp["uy"])
        B.run(6)
        tau, nst, st = B.events()
        assert st[1] == EVENT_FAILED
        assert st[0] == EVENT_RUNNING and st[2] == EVENT_RUNNING and nst[0] == 6 and nst[2] == 6
        # the healthy events evolved as if alone
        for ev, seed in ((0, 1), (2, 3)):
            ref = single_event(cfg, 24, 4.0, seed, 6)
            got = B.event_state(ev)
            for q in range(14):
                assert rel_err(got[q], ref[q]) <= 1e-13


def test_autotune_picks_a_compiled_variant(tmp_path):
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True, precision=A.PREC_MIXED)
    with Batch(cfg, [40, 64, 96, 50], tau0=cfg.tau0, dtau=cfg.dtau, tau_max=100.0, t_freeze_gev=0.0) as B:
        B.init_glauber(seeds=[0, 1, 2, 3], bimp=[3.0, 6.0, 9.0, 1.0])
        before = [B.event_state(e) for e in range(4)]
        cache = str(tmp_path / "tune.txt")
        ms = B.autotune(cache, probe_steps=8)
        assert ms > 0
        t = B.tuning()
        assert 0 <= t["variant"] <= 4 and t["steps_per_launch"] in (8, 32)
        # the trials leave the state and the clocks as they were
        tau, nst, st = B.events()
        assert np.all(nst == 0) and np.allclose(tau, cfg.tau0)
        for e in range(4):
            assert np.array_equal(B.event_state(e), before[e])
        # a second tuning with the same key reads the cache
        assert B.autotune(cache, probe_steps=8) < 0
        assert "=" in open(cache).read()


def test_per_event_observables():
    """eps_p of every batched event equals vh_eps_p of the same event stepped
    alone; eps_2 equals the energy-density eccentricity of its state"""
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True)
    sides, bimp = [30, 41, 26], [6.0, 9.0, 3.0]
    steps = 10
    with Batch(cfg, sides, tau0=cfg.tau0, dtau=cfg.dtau, tau_max=100.0, t_freeze_gev=0.0) as B:
        B.init_glauber(seeds=[4, 5, 6], bimp=bimp)
        ep0, e20 = B.observables()
        B.run(steps)
        ep, e2 = B.observables()
        states = [B.event_state(ev) for ev in range(3)]
    for ev, (side, b) in enumerate(zip(sides, bimp)):
        c = C.glauber_config(nx=side, ny=side, boost_invariant=True)
        with C.make_hydro(c, C.glauber_inputs(c, b=b, seed=4 + ev)) as H:
            assert abs(H.eps_p() - ep0[ev]) <= 1e-12 * max(abs(ep0[ev]), 1e-3)
            H.step(steps)
            assert abs(H.eps_p() - ep[ev]) <= 1e-12 * max(abs(ep[ev]), 1e-3)
        g = side + 6
        e = states[ev][0].reshape(g, g)[3:3 + side, 3:3 + side]
        yy, xx = np.meshgrid(np.arange(side) * 0.1, np.arange(side) * 0.1, indexing="ij")
        E = e.sum()
        xm, ym = (e * xx).sum() / E, (e * yy).sum() / E
        sxx = (e * xx * xx).sum() / E - xm * xm
        syy = (e * yy * yy).sum() / E - ym * ym
        sxy = (e * xx * yy).sum() / E - xm * ym
        want = np.sqrt((syy - sxx) ** 2 + 4 * sxy ** 2) / (sxx + syy)
        assert abs(e2[ev] - want) <= 1e-10 * want
    assert np.all(np.abs(ep0) < 1e-12)  # at rest with pi = 0: T^xx = T^yy = P


def test_barrier_timeout_is_reported_and_the_context_survives():
    """The persistent kernel's grid barrier gives up after a bounded wait: a
    launch where one block never arrives returns VH_E_TIMEOUT (no fault, no
    hang), and the same context then runs a batch normally"""
    import ctypes
    L = A.lib()
    sec = ctypes.c_double(-1.0)
    assert L.vh_batch_barrier_selftest(0, ctypes.byref(sec)) == A.OK
    assert 0 <= sec.value < 0.1
    assert L.vh_batch_barrier_selftest(1, ctypes.byref(sec)) == A.E_TIMEOUT
    assert b"timed out" in L.vh_batch_last_error(None)
    assert 0 < sec.value < 10, sec.value
    print("barrier wait gave up after %.3f s" % sec.value)
    assert L.vh_batch_barrier_selftest(2, None) == A.E_ARG
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True)
    with Batch(cfg, [24, 30], tau0=cfg.tau0, dtau=cfg.dtau, tau_max=100.0, t_freeze_gev=0.0) as B:
        B.init_glauber(seeds=[0, 1], bimp=[3.0, 6.0])
        B.run(4)
        tau, nst, st = B.events()
        assert np.all(st == EVENT_RUNNING) and np.all(nst == 4)
