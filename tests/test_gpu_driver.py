"""The C++ host driver against the Python path over the same C ABI: the
snapshots it writes (the reference's file names and layouts) are the bytes
vh_write gives after the same steps; and vh_get_primitive returns the state's
primitive fields with the dependent pi components consistent."""
import os
import subprocess

import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200 import build
from viral_b200 import configs as C

pytestmark = pytest.mark.gpu


def run_driver(args, tmp):
    out = os.path.join(tmp, "res")
    r = subprocess.run([build.build_driver(), *args, "--out", out, "--quiet"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return out


def test_gubser_snapshots_match_the_python_path(tmp_path):
    steps = 6
    out = run_driver(["--scenario", "gubser", "--nx", "33", "--ny", "33", "--steps", str(steps),
                      "--print-every", "0.03"], str(tmp_path))
    names = sorted(os.listdir(out))
    assert names == ["tau1.000fm.bin", "tau1.010fm.bin", "tau1.030fm.bin", "tau1.060fm.bin"], names
    cfg = C.gubser_config(nx=33, ny=33)
    with C.make_hydro(cfg, C.gubser_inputs(cfg)) as H:
        H.step(steps)
        mine = os.path.join(str(tmp_path), "py.bin")
        H.write(mine, A.WRITE_XY, 1)
    assert open(mine, "rb").read() == open(os.path.join(out, "tau1.060fm.bin"), "rb").read()


def test_glauber_snapshot_matches_the_python_path(tmp_path):
    steps = 5
    out = run_driver(["--scenario", "glauber", "--nx", "40", "--ny", "40", "--steps", str(steps), "--b", "6",
                      "--seed", "3", "--every", "2", "--print-every", "0.1"], str(tmp_path))
    cfg = C.glauber_config(nx=40, ny=40, boost_invariant=True)
    with C.make_hydro(cfg, C.glauber_inputs(cfg, b=6.0, seed=3)) as H:
        H.step(steps)
        mine = os.path.join(str(tmp_path), "py.bin")
        H.write(mine, A.WRITE_XY, 2)
    assert open(mine, "rb").read() == open(os.path.join(out, "tau0.700fm.bin"), "rb").read()


def test_driver_restart_continues_the_run(tmp_path):
    """--checkpoint after 8 steps, then --restart from it up to step 16: the
    final restart file and the last snapshot equal those of one 16-step run"""
    t = str(tmp_path)
    common = ["--scenario", "glauber", "--nx", "36", "--ny", "36", "--b", "5", "--seed", "1", "--print-every", "0.16"]
    whole, part = os.path.join(t, "whole"), os.path.join(t, "part")
    os.makedirs(whole), os.makedirs(part)
    run_driver(common + ["--steps", "16", "--checkpoint", os.path.join(t, "whole.ck")], whole)
    run_driver(common + ["--steps", "8", "--checkpoint", os.path.join(t, "half.ck")], part)
    run_driver(common + ["--steps", "16", "--restart", os.path.join(t, "half.ck"), "--checkpoint",
                         os.path.join(t, "resumed.ck")], part)
    assert open(os.path.join(t, "whole.ck"), "rb").read() == open(os.path.join(t, "resumed.ck"), "rb").read()
    snap = "tau0.920fm.bin"
    assert open(os.path.join(whole, "res", snap), "rb").read() == open(os.path.join(part, "res", snap), "rb").read()


def test_driver_navier_stokes_files(tmp_path):
    """--ns: beside each snapshot the Navier-Stokes file of NEWEST10's
    initialisation (res/NStau%2.3ffm.bin), the bytes vh_write gives"""
    out = run_driver(["--scenario", "gubser", "--nx", "33", "--ny", "33", "--steps", "3", "--print-every", "0.03",
                      "--ns"], str(tmp_path))
    names = sorted(os.listdir(out))
    assert "NStau1.000fm.bin" in names and "NStau1.030fm.bin" in names, names
    cfg = C.gubser_config(nx=33, ny=33)
    with C.make_hydro(cfg, C.gubser_inputs(cfg)) as H:
        first = os.path.join(str(tmp_path), "ns0.bin")
        H.write(first, A.WRITE_NS_XY, 1)
        H.step(3)
        last = os.path.join(str(tmp_path), "ns3.bin")
        H.write(last, A.WRITE_NS_XY, 1)
    assert open(first, "rb").read() == open(os.path.join(out, "NStau1.000fm.bin"), "rb").read()
    assert open(last, "rb").read() == open(os.path.join(out, "NStau1.030fm.bin"), "rb").read()


def test_driver_bjorken_temperature_file(tmp_path):
    """--scenario bjorken writes ./temp.txt as the reference's main loop
    does: per step the tau the step started from and the centre cell's
    T (fm^-1) x 0.1973 / 1000, until tau > 10 fm/c"""
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_bjorken.npz"))
    r = subprocess.run([build.build_driver(), "--scenario", "bjorken", "--quiet"], capture_output=True, text=True,
                       timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    rows = np.loadtxt(os.path.join(str(tmp_path), "temp.txt"))
    tau, nsteps = 0.6, 0
    while True:  # the reference's loop: tau += ts, break once tau > 10
        tau += 0.01
        nsteps += 1
        if tau > 10:
            break
    assert rows.shape == (nsteps, 2)
    assert np.allclose(rows[:, 0], 0.6 + 0.01 * np.arange(nsteps), atol=1e-9)
    m = min(nsteps, len(g["temp"]))
    assert np.allclose(rows[:m, 1], g["temp"][:m] * 0.1973 / 1000, rtol=1e-5, atol=0)


def test_driver_cold_plasma_snapshot(tmp_path):
    """--scenario gubser --cold-plasma: the snapshot after 4 steps is the
    Python path's (vh_profile_gubser_cold, the source without -pi/tau_pi)"""
    from viral_b200.hydro import Hydro, profile_gubser_cold
    out = run_driver(["--scenario", "gubser", "--cold-plasma", "--nx", "33", "--ny", "33", "--steps", "4",
                      "--print-every", "0.04"], str(tmp_path))
    cfg = C.gubser_config(nx=33, ny=33)
    cfg.cold_plasma = True
    with Hydro(cfg) as H:
        e, ux, uy, pi5, pu = profile_gubser_cold(33, 33, cfg.dx, cfg.dy, 1.0, cfg.tau0, cfg.dtau, 1.21, cfg.eos_a)
        H.init_profile(cfg.tau0, e, ux, uy, None, pu, A.PI_GIVEN, pi5)
        H.step(4)
        mine = os.path.join(str(tmp_path), "py.bin")
        H.write(mine, A.WRITE_XY, 1)
    assert open(mine, "rb").read() == open(os.path.join(out, "tau1.040fm.bin"), "rb").read()


def test_get_primitive():
    cfg = C.gubser_config(nx=21, ny=21)
    with C.make_hydro(cfg, C.gubser_inputs(cfg)) as H:
        H.step(3)
        tau = H.tau
        s = H.get_state()
        p = H.get_primitive()
    assert np.array_equal(p["e"], s[0]) and np.array_equal(p["u"], s[1:5])
    assert np.allclose(p["P"], s[0] / 3, rtol=1e-15)
    assert np.allclose(p["T"], (s[0] / cfg.eos_a) ** 0.25, rtol=1e-14)
    pi = p["pi"]
    assert np.array_equal(pi[4], s[5]) and np.array_equal(pi[7], s[6]) and np.array_equal(pi[5], s[7])
    # transversality u_mu pi^{mu nu} = 0 and tracelessness g_{mu nu} pi^{mu nu} = 0, metric diag(1,-1,-1,-tau^2)
    u = p["u"]
    g = np.array([1.0, -1.0, -1.0, -tau * tau])
    full = np.zeros((4, 4, pi.shape[1]))
    idx = {(0, 0): 0, (0, 1): 1, (0, 2): 2, (0, 3): 3, (1, 1): 4, (1, 2): 5, (1, 3): 6, (2, 2): 7, (2, 3): 8, (3, 3): 9}
    for (a, b), q in idx.items():
        full[a, b] = pi[q]
        full[b, a] = pi[q]
    scale = np.abs(pi).max()
    for nu in range(4):
        assert np.abs(sum(g[m] * u[m] * full[m, nu] for m in range(4))).max() <= 1e-12 * scale
    assert np.abs(sum(g[m] * full[m, m] for m in range(4))).max() <= 1e-12 * scale


def test_shock_tube_scenario_matches_the_reference(tmp_path):
    """vh_run --scenario shocktube, 20 steps: the full-grid snapshot holds the
    reference's own state of its Cartesian default block"""
    from helpers import shock_tube_fixture
    g, ocfg, f = shock_tube_fixture()
    out = run_driver(["--scenario", "shocktube", "--steps", "20", "--print-every", "0.2"], str(tmp_path))
    snap = np.fromfile(os.path.join(out, "tau0.200fm.bin"), dtype=np.float64).reshape(-1, 12)
    nx, ny, nz = ocfg.nx, ocfg.ny, ocfg.nz
    # records x outer, y, then z inner; fixture cells are interior cells in (k, j, i) order
    e = snap[:, 0].reshape(nx, ny, nz).transpose(2, 1, 0).ravel()
    ref = g["state"][0]
    assert np.max(np.abs(e - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("every", [1, 2])
def test_seventeen_variable_snapshots(tmp_path, every):
    """VH_WRITE_XY17 / VH_WRITE_FULL17 (NEWEST10/write.h): e, T, P, v, the ten
    pi^{mu nu} and Pi per cell, x outer, y, then eta"""
    cfg = C.glauber_config(nx=12, ny=10, nz=8, boost_invariant=False)
    with C.make_hydro(cfg, C.glauber_inputs(cfg, b=4.0, seed=1)) as H:
        H.step(3)
        s = H.get_state()
        p = H.get_primitive()
        xy = os.path.join(str(tmp_path), "xy.bin")
        full = os.path.join(str(tmp_path), "full.bin")
        H.write(xy, A.WRITE_XY17, every)
        H.write(full, A.WRITE_FULL17, every)
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz

    def rec(i, j, k):
        c = (k * gy + j) * gx + i
        u0 = s[1, c]
        return [s[0, c], p["T"][c], p["P"][c], s[2, c] / u0, s[3, c] / u0, s[4, c] / u0, *p["pi"][:, c], 0.0]

    # T and P come from the EOS at e on the host (the reference's FT and EOS
    # on its cells); the device's interpolation may round differently
    def same(got, want):
        want = np.array(want)
        cols = [0, 3, 4, 5, *range(6, 17)]
        assert np.array_equal(got[:, cols], want[:, cols])
        assert np.allclose(got[:, 1:3], want[:, 1:3], rtol=1e-14, atol=0)

    want_xy = [rec(i, j, (gz - 1) // 2) for i in range(3, 3 + cfg.nx, every) for j in range(3, 3 + cfg.ny, every)]
    same(np.fromfile(xy, dtype=np.float64).reshape(-1, 17), want_xy)
    want_full = [rec(i, j, k) for i in range(3, 3 + cfg.nx, every) for j in range(3, 3 + cfg.ny, every)
                 for k in range(3, 3 + cfg.nz)]
    same(np.fromfile(full, dtype=np.float64).reshape(-1, 17), want_full)
