"""GPU step versus the oracle (FP64 mode) through the C ABI.

Tolerances: the FP64 GPU step and the oracle differ only by rounding
(fused multiply-adds, division and pow implementations), so single-stage
terms agree to 1e-12 relative (max norm over the grid) and full runs to
1e-10 relative, the FP64 bar of the reference comparison.
"""
import numpy as np
import pytest

from conftest import rel_err
from helpers import interior_mask, oracle_config, oracle_from_inputs, smooth_inputs
from pyoracle import Oracle
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Config, Hydro

pytestmark = pytest.mark.gpu

STAGE_TOL = 1e-12
RUN_TOL = 1e-10


def milne3d(**kw):
    base = dict(nx=20, ny=18, nz=12, boost_invariant=False, dx=0.1, dy=0.1, dz=0.1, tau0=1.3, dtau=0.01,
                eos_kind=A.EOS_CONFORMAL, eos_a=13.899692864867510, etas0=1 / (4 * np.pi))
    base.update(kw)
    return Config(**base)


# field groups normalised together: e; u^mu; pi^{mu nu}; T^{tau mu}; prevu
GROUPS = [(0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)]


def compare_states(a, b, tol, fields=range(14), mask=None):
    """Max |a-b| of each field over the largest |b| of its tensor group
    (a component that stays near zero is compared on the scale of its tensor)."""
    errs = {}
    for grp in GROUPS:
        scale = max(float(np.max(np.abs(b[q] if mask is None else b[q][mask]))) for q in grp)
        for q in grp:
            if q not in fields:
                continue
            x, y = (a[q], b[q]) if mask is None else (a[q][mask], b[q][mask])
            d = float(np.max(np.abs(x - y)))
            errs[q] = 0.0 if d == 0 else d / (scale if scale > 0 else 1.0)
    worst = max(errs.values())
    assert worst <= tol, f"max rel err {worst:.3e} > {tol:.1e}: {errs}"
    return worst


@pytest.mark.parametrize("cfgkw", [
    dict(),
    dict(boost_invariant=True, nz=1),
    dict(coords=A.COORD_CARTESIAN, tau0=1.0),
    dict(recon=A.RECON_MINMOD),
    dict(eos_kind=A.EOS_TABLE, eos_table=C.eos_table(), etas0=0.08, etas1=1.0),
    dict(gubser_mirror=True, taupi_kind=A.TAUPI_5_ETA_OVER_EPP, etas0=0.2, boost_invariant=True, nz=1),
])
def test_stage_terms_match_oracle(cfgkw):
    cfg = milne3d(**cfgkw)
    f = smooth_inputs(cfg, cfg.tau0, seed=11)
    O = Oracle(oracle_config(cfg))
    O.set_state(f)
    so, ro, do = O.stage_terms(cfg.tau0, cfg.dtau)
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        rg, sg, dg = H.debug_stage_terms()
    m = interior_mask(cfg)
    for l in range(9):
        assert rel_err(rg[l][m], ro[l][m]) <= STAGE_TOL, f"flux divergence {l}"
        assert rel_err(sg[l][m], so[l][m]) <= STAGE_TOL, f"source {l}"
    assert rel_err(dg[:, m], do[:, m]) <= STAGE_TOL


@pytest.mark.parametrize("cfgkw", [
    dict(),
    dict(boost_invariant=True, nz=1),
    dict(coords=A.COORD_CARTESIAN, tau0=1.0),
    dict(recon=A.RECON_MINMOD),
    dict(eos_kind=A.EOS_TABLE, eos_table=C.eos_table(), etas0=0.08, etas1=1.0),
])
def test_steps_match_oracle(cfgkw):
    cfg = milne3d(**cfgkw)
    f = smooth_inputs(cfg, cfg.tau0, seed=5)
    O = Oracle(oracle_config(cfg))
    O.set_state(f)
    tau = cfg.tau0
    for _ in range(4):
        assert O.step(tau, cfg.dtau) == 0
        tau += cfg.dtau
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        H.step(4)
        g = H.get_state()
        assert abs(H.tau - tau) < 1e-12
    compare_states(g, O.get_state(), 1e-11, fields=range(18))


def test_gubser_run_matches_oracle():
    """The boost-invariant Gubser test (129x129, NS pi, mirrored ghosts),
    50 steps of the GPU step against the oracle (all 300 steps to tau = 4:
    tests/test_gpu_gubser.py)."""
    cfg = C.gubser_config()
    inp = C.gubser_inputs(cfg)
    O = oracle_from_inputs(cfg, inp)
    with C.make_hydro(cfg, inp) as H:
        compare_states(H.get_state(), O.get_state(), STAGE_TOL, fields=range(18))
        tau = cfg.tau0
        for _ in range(50):
            assert O.step(tau, cfg.dtau) == 0
            tau += cfg.dtau
        H.step(50)
        compare_states(H.get_state(), O.get_state(), RUN_TOL, fields=range(18))
        assert abs(H.max_temperature() - O.max_temp_gev()) <= 1e-12 * O.max_temp_gev()


def test_glauber_boost_invariant_matches_oracle():
    cfg = C.glauber_config(nx=64, ny=64, boost_invariant=True)
    inp = C.glauber_inputs(cfg, b=7.0, seed=3)
    O = oracle_from_inputs(cfg, inp)
    with C.make_hydro(cfg, inp) as H:
        tau = cfg.tau0
        for _ in range(40):
            assert O.step(tau, cfg.dtau) == 0
            tau += cfg.dtau
        H.step(40)
        compare_states(H.get_state(), O.get_state(), RUN_TOL, fields=range(18))


def test_glauber_3d_matches_oracle():
    cfg = C.glauber_config(nx=40, ny=36, nz=12, deta=0.25)
    inp = C.glauber_inputs(cfg, b=7.0, seed=0)
    O = oracle_from_inputs(cfg, inp)
    with C.make_hydro(cfg, inp) as H:
        tau = cfg.tau0
        for _ in range(10):
            assert O.step(tau, cfg.dtau) == 0
            tau += cfg.dtau
        H.step(10)
        compare_states(H.get_state(), O.get_state(), RUN_TOL, fields=range(18))


def test_mixed_precision_tracks_fp64():
    """FP32 state/fluxes/sources with the FP64 root-find stay close to the
    FP64 step on a smooth event (relative max error in e, u, pi)."""
    cfg64 = C.glauber_config(nx=64, ny=64, boost_invariant=True)
    cfg32 = C.glauber_config(nx=64, ny=64, boost_invariant=True, precision=A.PREC_MIXED)
    inp = C.glauber_inputs(cfg64, b=7.0, seed=1)
    with C.make_hydro(cfg64, inp) as H64, C.make_hydro(cfg32, inp) as H32:
        H64.step(40)
        H32.step(40)
        a, b = H32.get_state(), H64.get_state()
    m = interior_mask(cfg64)
    assert rel_err(a[0][m], b[0][m]) < 1e-4
    for q in (2, 3):
        assert rel_err(a[q][m], b[q][m]) < 1e-3
    for q in (5, 6, 7):
        assert rel_err(a[q][m], b[q][m]) < 1e-2


def test_reductions():
    cfg = C.gubser_config(nx=33, ny=33)
    inp = C.gubser_inputs(cfg)
    O = oracle_from_inputs(cfg, inp)
    f = O.get_state()
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        assert abs(H.max_temperature() - O.max_temp_gev()) <= 1e-13
        sums = H.conservation_sums()
        m = interior_mask(cfg)
        ref = [np.sum(cfg.tau0 * f[10 + l][m]) * cfg.dx * cfg.dy for l in range(4)]
        for l in range(4):
            assert abs(sums[l] - ref[l]) <= 1e-12 * max(1.0, abs(ref[0]))
        a, dt = H.cfl()
        assert 0 < a < 1 and abs(dt - cfg.dx / (8 * a)) < 1e-15


def test_step_errors_are_reported():
    """A superluminal T^{tau mu} makes the root-find fail; the call returns
    an error status instead of exiting, and the handle stays usable."""
    cfg = milne3d(boost_invariant=True, nz=1)
    f = smooth_inputs(cfg, cfg.tau0, seed=2)
    f[11] *= 50.0  # |T^{tau x}| >> T^{tau tau} in every cell
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        with pytest.raises(A.VhError) as ei:
            H.step(1)
        assert ei.value.code in (A.E_ROOTFIND, A.E_CAUSALITY, A.E_NEG_ENERGY)
        good = smooth_inputs(cfg, cfg.tau0, seed=2)
        H.set_state(good, cfg.tau0)
        H.step(1)


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_cartesian_shock_tube_matches_reference(precision):
    """The reference's Cartesian shock tube (its default TXYZ5 block, 10x10x101,
    e = 16 / 1 fm^-4 across z = 0), 20 steps, against the reference's own
    state (tests/golden/ref_cart_3d_shock.npz): FP64 within 1e-10, the mixed
    step within 1e-4 of each tensor's scale"""
    from helpers import shock_tube_fixture
    g, ocfg, f = shock_tube_fixture()
    dx, dy, dz, factor, gevfm = (float(v) for v in g["consts"])
    cfg = Config(nx=ocfg.nx, ny=ocfg.ny, nz=ocfg.nz, boost_invariant=False, coords=A.COORD_CARTESIAN,
                 precision=precision, dx=dx, dy=dy, dz=dz, tau0=0.0, dtau=float(g["ts"]), eos_kind=A.EOS_CONFORMAL,
                 eos_a=factor, etas0=0.01 / (4 * np.pi), etas1=0.0, hbarc=gevfm, taupi_kind=A.TAUPI_15_ETA_OVER_P)
    with Hydro(cfg) as H:
        H.set_state(f, 0.0)
        H.step(int(g["steps"]))
        s = H.get_state()
    c = g["cells"]
    tol = RUN_TOL if precision == A.PREC_FP64 else 1e-4
    worst = 0.0
    for grp in GROUPS:
        grp = [q for q in grp if q < 14]
        if not grp:
            continue
        scale = float(np.max(np.abs(g["state"][grp])))
        err = float(np.max(np.abs(s[grp][:, c] - g["state"][grp]))) / (scale if scale > 0 else 1.0)
        worst = max(worst, err)
    print("shock tube, precision %d: max error %.2e" % (precision, worst))
    assert worst <= tol


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_bjorken_scenario_matches_reference(precision):
    """The reference's Bjorken scenario, 940 steps to tau = 10 fm/c: the
    centre temperature after every step against the compiled reference's
    (tests/golden/ref_bjorken.npz); FP64 to 1e-12, mixed to 1e-5"""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_bjorken.npz"))
    cfg = C.bjorken_config(precision=precision)
    c = int(g["centre"])
    temps = []
    with C.make_hydro(cfg, C.bjorken_inputs(cfg)) as H:
        for _ in range(int(g["steps"])):
            H.step(1)
            temps.append(H.get_primitive()["T"][c])
        final = H.get_state()[:, c]
    err = float(np.max(np.abs(np.array(temps) - g["temp"]) / g["temp"]))
    print("Bjorken %s: max rel err of T over 940 steps %.2e" % ("fp64" if precision == A.PREC_FP64 else "mixed", err))
    assert err <= (1e-12 if precision == A.PREC_FP64 else 1e-5)
    if precision == A.PREC_FP64:
        assert np.max(np.abs(final - g["final"])) <= 1e-12 * np.max(np.abs(g["final"]))


@pytest.mark.late
@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
def test_cartesian_bjorken_block_stays_at_rest(precision):
    """The reference's Cartesian Bjorken block (TXYZ5, 10x10x41, 100 steps
    from t = 0.6; tests/golden/ref_cart_bjorken.npz): the compiled reference
    keeps the uniform fluid at rest bitwise.  FP64 to 1e-12 (the root-find
    may move e by an ulp per stage), the mixed mode to its FP32 state
    (1e-6) (late: newer than the rest of this file)"""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cart_bjorken.npz"))
    cfg = C.cart_bjorken_config(precision=precision)
    assert cfg.gdims() == tuple(int(v) for v in g["dims"][:3])
    with C.make_hydro(cfg, C.cart_bjorken_inputs(cfg)) as H:
        start = H.get_state()
        H.step(int(g["steps"]))
        end = H.get_state()
        assert H.tau == pytest.approx(float(g["t0"]) + int(g["steps"]) * float(g["ts"]), abs=1e-12)
    tol = 1e-12 if precision == A.PREC_FP64 else 1e-6
    scale = np.abs(g["final"]).max()
    assert np.abs(end[:, int(g["centre"])] - g["final"]).max() <= tol * scale
    assert np.abs(end[:14] - start[:14]).max() <= tol * scale


@pytest.mark.late
def test_bench_workload_matches_oracle():
    """The benchmarked workload itself (bench.py's glauber_161x161x41: the
    3+1D MC-Glauber event, 1,062,761 interior cells, FP64) against the
    oracle (its cell loops on the host's cores) after 2 and after 70 steps
    (tau = 2 fm/c: before the event's trajectories separate, any rounding
    difference grows by some 4 % per step later on), every field on the
    whole ghost-inclusive grid; and the mixed mode's two steps against the
    FP64 ones (late: newer than the rest of this file)"""
    import bench
    cfg, inp, _ = bench.build_workload("glauber_161x161x41", "fp64")
    O = oracle_from_inputs(cfg, inp)
    with C.make_hydro(cfg, inp) as H:
        compare_states(H.get_state(), O.get_state(), STAGE_TOL, fields=range(18))
        tau, done = cfg.tau0, 0
        for k in (2, 70):
            for _ in range(k - done):
                assert O.step(tau, cfg.dtau) == 0
                tau += cfg.dtau
            H.step(k - done)
            done = k
            st = H.get_state()
            worst = compare_states(st, O.get_state(), RUN_TOL, fields=range(18))
            print("161x161x41, %d steps: max group-relative error against the oracle %.2e" % (k, worst))
            if k == 2:
                s64 = st
    cfg32, inp32, _ = bench.build_workload("glauber_161x161x41", "mixed")
    with C.make_hydro(cfg32, inp32) as H:
        H.step(2)
        s32 = H.get_state()
    m = interior_mask(cfg)
    assert rel_err(s32[0][m], s64[0][m]) < 1e-4  # the bounds of test_mixed_precision_tracks_fp64
    for q in (1, 2, 3, 4):
        assert rel_err(s32[q][m], s64[q][m]) < 1e-3


@pytest.mark.parametrize("cfgkw", [dict(), dict(coords=A.COORD_CARTESIAN, tau0=1.0)])
def test_get_conserved(cfgkw):
    """the reference's Var: tau T^{tau mu} (T^{t mu} in Cartesian), pi, 0"""
    cfg = milne3d(**cfgkw)
    f = smooth_inputs(cfg, cfg.tau0, seed=2)
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        H.step(2)
        s, tau, var = H.get_state(), H.tau, H.get_conserved()
    t = 1.0 if cfg.coords == A.COORD_CARTESIAN else tau
    assert np.array_equal(var[:4], t * s[10:14])
    assert np.array_equal(var[4:9], s[5:10])
    assert np.all(var[9] == 0)


def test_cold_plasma_gubser_flow():
    """the reference's cold-plasma test (the shear source without -pi/tau_pi):
    the GPU against the oracle over 10 steps, and against the closed form
    to tau = 1.5 fm/c on a 129 x 129 grid"""
    from test_cold_plasma_cpu import A_CONF, closed_form_T, cold_config, radius, run_oracle
    from viral_b200.hydro import profile_gubser_cold

    def start(H, cfg):
        e, ux, uy, pi5, pu = profile_gubser_cold(cfg.nx, cfg.ny, cfg.dx, cfg.dy, 1.0, cfg.tau0, cfg.dtau, 1.21, A_CONF)
        H.init_profile(cfg.tau0, e, ux, uy, None, pu, A.PI_GIVEN, pi5)

    cfg = cold_config(41, 0.1, 0.01)
    ref, _ = run_oracle(cfg, 10)
    with Hydro(cfg) as H:
        start(H, cfg)
        H.step(10)
        compare_states(H.get_state(), ref, RUN_TOL, fields=range(18))
    cfg = cold_config(129, 0.1, 0.01)
    with Hydro(cfg) as H:
        start(H, cfg)
        H.step(50)
        s, tau = H.get_state(), H.tau
    r = radius(cfg)
    m = r < 2.0
    err = np.max(np.abs((s[0][m] / A_CONF) ** 0.25 / closed_form_T(r[m], tau) - 1))
    print("cold plasma on the GPU to tau = %.2f: T within %.2e of the closed form" % (tau, err))
    assert err <= 6e-4


@pytest.mark.parametrize("cfgkw", [
    dict(nx=3, ny=3, nz=1, boost_invariant=True),
    dict(nx=3, ny=4, nz=3),
    dict(nx=3, ny=3, nz=3, coords=A.COORD_CARTESIAN, tau0=1.0),
])
def test_smallest_grids_match_oracle(cfgkw):
    """three interior cells per axis, the minimum vh_create accepts: every
    stencil reaches into the ghosts on both sides"""
    cfg = milne3d(**cfgkw)
    f = smooth_inputs(cfg, cfg.tau0, seed=9)
    O = Oracle(oracle_config(cfg))
    O.set_state(f)
    tau = cfg.tau0
    for _ in range(3):
        assert O.step(tau, cfg.dtau) == 0
        tau += cfg.dtau
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        H.step(3)
        compare_states(H.get_state(), O.get_state(), 1e-11, fields=range(18))


@pytest.mark.late
def test_mixed_precision_near_its_weno_range():
    """The mixed mode's FP32 WENO weights divide once per face pair by a
    number of order (stencil difference)^8, which overflows FP32 above
    differences of about 1e4 (include/vh.h).  A hot spot of 5000 fm^-4
    (about 1000 GeV/fm^3) and 0.3 fm width at tau = 0.6 fm/c, differences of
    a few thousand per cell, stays finite and tracks the FP64 step to FP32
    rounding over 10 steps (late: newer than the rest of this file)."""
    cfg64 = C.glauber_config(nx=48, ny=48, boost_invariant=True)
    gx, gy, _ = cfg64.gdims()
    idx = np.arange(gx * gy)
    x = (idx % gx - 3 - 24) * cfg64.dx
    y = (idx // gx - 3 - 24) * cfg64.dy
    e = 1.0 + 5000.0 * np.exp(-(x * x + y * y) / (2 * 0.3 ** 2))
    z = np.zeros_like(e)
    inp = dict(tau=cfg64.tau0, e=e, ux=z, uy=z, ueta=None, prevu=None, pi_mode=A.PI_ZERO)
    out = []
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        cfg = C.glauber_config(nx=48, ny=48, boost_invariant=True, precision=prec)
        with C.make_hydro(cfg, inp) as H:
            H.step(10)
            out.append(H.get_state())
    m = interior_mask(cfg64)
    assert np.all(np.isfinite(out[1]))
    assert rel_err(out[1][0][m], out[0][0][m]) < 1e-4
    for q in (1, 2, 3):
        assert rel_err(out[1][q][m], out[0][q][m]) < 1e-3
