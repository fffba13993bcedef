"""CPU checks of the C ABI library: it loads without a GPU, exports every
entry point include/vh.h declares, and its host-side input generators are
deterministic and physically sane.  No device computation runs here."""
import os
import re
import subprocess

import numpy as np
import pytest

from viral_b200 import _abi as A
from viral_b200 import hydro as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "vh.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vh_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_expected_surface():
    syms = declared_symbols()
    for s in ("vh_create", "vh_destroy", "vh_set_state", "vh_get_state", "vh_init_profile", "vh_step",
              "vh_max_temperature", "vh_write", "vh_step_static"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = A.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (vh_[a-z0-9_]+)$", out, flags=re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    L = A.lib()  # loads without a GPU
    for name, _, _ in A.SIGNATURES:
        assert hasattr(L, name)
    assert {n for n, _, _ in A.SIGNATURES} == set(declared_symbols())


def test_create_rejects_bad_config_without_gpu():
    cfg = H.Config(nx=2, ny=10)  # too few cells: rejected before any device call
    with pytest.raises(A.VhError) as e:
        H.Hydro(cfg)
    assert e.value.code == A.E_ARG


def test_create_rejects_bad_relaxation_time_without_gpu():
    for kw in (dict(taupi_kind=A.TAUPI_CONST, taupi_const=0.0), dict(taupi_kind=7)):
        with pytest.raises(A.VhError) as e:
            H.Hydro(H.Config(nx=10, ny=10, **kw))
        assert e.value.code == A.E_ARG


def test_eos_table_properties():
    t = H.eos_table_synthetic(2000, 1e-3, 500.0)
    e, p, cs2, T = t
    hc = H.HBARC
    assert np.all(np.diff(e) > 0) and np.all(np.diff(p) > 0) and np.all(np.diff(T) > 0)
    # log spacing and range in GeV/fm^3
    assert abs(e[0] * hc - 1e-3) < 1e-15 and abs(e[-1] * hc - 500.0) < 1e-10
    assert np.allclose(np.diff(np.log(e)), np.log(5e5) / 1999, rtol=1e-9)
    # c_s^2 formula and anchors
    eg = e * hc
    assert np.allclose(cs2, 1 / 3 - 0.2 * np.exp(-0.5 * np.log(eg / 0.5) ** 2), rtol=1e-14)
    assert abs(p[0] - cs2[0] * e[0]) < 1e-18
    assert abs(e[-1] - H.A_QGP * T[-1] ** 4) < 1e-9 * e[-1]
    # thermodynamic consistency: dP/de = cs2 and d ln T / de = cs2/(e+P)
    dp = np.diff(p) / np.diff(e)
    assert np.allclose(dp, 0.5 * (cs2[1:] + cs2[:-1]), rtol=2e-4)
    dlt = np.diff(np.log(T)) / np.diff(e)
    assert np.allclose(dlt, 0.5 * ((cs2 / (e + p))[1:] + (cs2 / (e + p))[:-1]), rtol=2e-3)


def test_gubser_profile():
    e, ux, uy, pu = H.profile_gubser(129, 129, 0.1, 0.1, q=1.0, tau0=1.0, dtau=0.01, t0_gev=0.6)
    g = 135
    E = e.reshape(g, g)
    c = g // 2
    assert abs((E[c, c] / H.A_QGP) ** 0.25 * H.HBARC - 0.6) < 1e-12
    assert np.allclose(E, E.T) and np.allclose(E, E[::-1, :]) and np.allclose(E, E[:, ::-1])
    UX = ux.reshape(g, g)
    assert np.allclose(UX, -UX[:, ::-1]) and UX[c, c] == 0.0
    # u^perp = sinh(kappa), tanh(kappa) = 2 q^2 tau r / (1 + q^2 tau^2 + q^2 r^2)
    x = (np.arange(g) - 3 - 64) * 0.1
    r = abs(x[c + 10])
    assert abs(UX[c, c + 10] - np.sinh(np.arctanh(2 * r / (2 + r * r)))) < 1e-14
    P = pu.reshape(4, g, g)
    assert np.allclose(P[0] ** 2, 1 + P[1] ** 2 + P[2] ** 2, rtol=1e-14)


def test_glauber_profile_deterministic_and_scaled():
    a, n1 = H.profile_glauber(64, 64, 1, True, 0.1, 0.1, 0.25, seed=3, efloor_gev=0.04)
    b, n2 = H.profile_glauber(64, 64, 1, True, 0.1, 0.1, 0.25, seed=3, efloor_gev=0.04)
    c, n3 = H.profile_glauber(64, 64, 1, True, 0.1, 0.1, 0.25, seed=4, efloor_gev=0.04)
    assert n1 == n2 and np.array_equal(a, b)
    assert not np.array_equal(a, c)
    E = a.reshape(70, 70)[3:67, 3:67]
    assert abs(E.max() * H.HBARC - 40.0) < 1e-9
    assert a.min() * H.HBARC >= 0.04 - 1e-15
    # Pb+Pb at b = 7 fm: a few hundred participants
    assert 100 < n1 < 416
    _, n0 = H.profile_glauber(32, 32, 1, True, 0.1, 0.1, 0.25, b=0.0, seed=1)
    _, n12 = H.profile_glauber(32, 32, 1, True, 0.1, 0.1, 0.25, b=12.0, seed=1)
    assert n0 > n12


def test_glauber_eta_profile():
    e, _ = H.profile_glauber(16, 16, 41, False, 0.1, 0.1, 0.25, seed=0, efloor_gev=0.0)
    E = e.reshape(47, 22, 22)
    col = E[:, 11, 11]
    eta = (np.arange(47) - 3 - 20) * 0.25
    flat = np.abs(eta) <= 1.5
    assert np.allclose(col[flat], col[flat][0])
    tail = ~flat
    expect = col[flat][0] * np.exp(-0.5 * (np.abs(eta[tail]) - 1.5) ** 2 / 1.3 ** 2)
    assert np.allclose(col[tail], expect, rtol=1e-12)
