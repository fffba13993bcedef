"""The Navier-Stokes shear tensor through the C ABI (vh_get_ns_pi, the
VH_WRITE_NS_XY snapshot) against the oracle's ten-component 2 eta sigma,
which the CPU tests pin to NEWEST10's own CalcNS."""
import os

import numpy as np
import pytest

from helpers import interior_mask, oracle_config, smooth_inputs
from pyoracle import Oracle
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Config, Hydro

pytestmark = pytest.mark.gpu


def cfg3d(**kw):
    base = dict(nx=20, ny=18, nz=12, boost_invariant=False, dx=0.1, dy=0.1, dz=0.1, tau0=1.3, dtau=0.01,
                eos_kind=A.EOS_CONFORMAL, eos_a=13.899692864867510, etas0=1 / (4 * np.pi))
    base.update(kw)
    return Config(**base)


def scaled_err(a, b):
    """max |a - b| over the largest |b| of the whole tensor"""
    s = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(a - b)))
    return 0.0 if d == 0 else d / (s if s > 0 else 1.0)


@pytest.mark.parametrize("cfgkw", [
    dict(),
    dict(boost_invariant=True, nz=1),
    dict(coords=A.COORD_CARTESIAN, tau0=1.0),
    dict(eos_kind=A.EOS_TABLE, eos_table=C.eos_table(), etas0=0.08, etas1=1.0),
])
def test_ns_pi_matches_oracle(cfgkw):
    """after two steps of a smooth viscous state: FP64 to rounding, the mixed
    mode (derivatives of the FP32 state in FP32) to 1e-4 of the tensor"""
    cfg = cfg3d(**cfgkw)
    f = smooth_inputs(cfg, cfg.tau0, seed=4)
    m = interior_mask(cfg)
    for precision, tol in ((A.PREC_FP64, 1e-12), (A.PREC_MIXED, 1e-4)):
        c = cfg3d(precision=precision, **cfgkw)
        with Hydro(c) as H:
            H.set_state(f, c.tau0)
            H.step(2)
            s, tau = H.get_state(), H.tau
            got = H.get_ns_pi()
        O = Oracle(oracle_config(cfg))
        O.set_state(s)
        want = O.ns_pi10(tau, cfg.dtau)
        err = scaled_err(got[:, m], want[:, m])
        print("NS pi %s %s: %.2e" % (cfgkw, "fp64" if precision == A.PREC_FP64 else "mixed", err))
        assert err <= tol
        # transverse (pi^{mu nu} u_nu = 0) and traceless (g_{mu nu} pi^{mu nu} = 0)
        if precision == A.PREC_FP64:
            t2 = 1.0 if cfg.coords == A.COORD_CARTESIAN else tau * tau
            g = np.array([1.0, -1.0, -1.0, -t2])
            P = np.zeros((4, 4, s.shape[1]))
            for q, (a, b) in enumerate([(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3),
                                        (3, 3)]):
                P[a, b] = P[b, a] = got[q]
            u = s[1:5]
            scale = np.max(np.abs(got[:, m]))
            for a in range(4):
                assert np.max(np.abs(sum(P[a, b] * g[b] * u[b] for b in range(4))[m])) <= 1e-12 * scale * 10
            assert np.max(np.abs(sum(g[a] * P[a, a] for a in range(4))[m])) <= 1e-12 * scale * 10


def test_ns_snapshot_layout(tmp_path):
    """VH_WRITE_NS_XY: 11 doubles per kept cell of the central eta slice,
    x outer, y inner, the ten components then a zero bulk part"""
    cfg = cfg3d()
    f = smooth_inputs(cfg, cfg.tau0, seed=9)
    path = str(tmp_path / "NStau1.300fm.bin")
    with Hydro(cfg) as H:
        H.set_state(f, cfg.tau0)
        ns = H.get_ns_pi()
        H.write(path, A.WRITE_NS_XY, 2)
    gx, gy, gz = cfg.gdims()
    k0 = (gz - 1) // 2
    rec = []
    for i in range(3, 3 + cfg.nx, 2):
        for j in range(3, 3 + cfg.ny, 2):
            c = (k0 * gy + j) * gx + i
            rec.append(np.concatenate([ns[:, c], [0.0]]))
    assert os.path.getsize(path) == len(rec) * 11 * 8
    assert np.array_equal(np.fromfile(path, dtype=np.float64), np.concatenate(rec))
