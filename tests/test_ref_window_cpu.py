"""The reference's table-EOS window builds (oracle/Makefile: the GINIT
scenario block of NEWEST5/maindef.h:240-295 with its s95p hooks on a run-time
table, ref_shim/eos_table_s95p.h), which time the reference's CPU step on
windows of the benchmark workloads, against the oracle on the same window:
the shim's EOS lookup and the block's transport (eta = s/4pi,
tau_pi = 1.5 eta/P) must give the oracle's step."""
import math
import os

import numpy as np
import pytest

from pyoracle import Oracle, OracleConfig, RefBuild, smooth_state
from viral_b200 import configs as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def _have(v):
    return os.path.exists(os.path.join(REF, f"libref_{v}.so"))


@pytest.mark.parametrize("variant", ["window_3d", "window_lbi"])
def test_window_build_steps_like_the_oracle(variant):
    if not _have(variant):
        pytest.skip("the reference's CPU builds are absent (oracle/Makefile)")
    R = RefBuild(variant)
    R.set_eos_table(C.eos_table())
    x, y, z = R.coords()
    tau, ts = 0.6, 0.02
    f = smooth_state(x, y, z, tau, ts, seed=3)
    if R.boost_invariant:
        for q in (4, 8, 9, 17):
            f[q] = 0.0
        for q in (1, 14):
            f[q] = np.sqrt(1 + f[q + 1] ** 2 + f[q + 2] ** 2)
    ocfg = OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=1 if R.boost_invariant else R.gz - 6,
                        boost_invariant=R.boost_invariant, dx=R.dx, dy=R.dy, dz=R.dz, eos_kind=1,
                        eos_table=C.eos_table(), etas0=1 / (4 * math.pi), taupi_kind=0)
    O = Oracle(ocfg)
    O.set_state(f)
    O.fill_tmunu(tau)
    R.set_state(O.get_state())
    for _ in range(2):
        R.step(tau, ts)
        assert O.step(tau, ts) == 0
        tau += ts
    a, b = R.get_state(), O.get_state()
    for g in ((0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13)):
        d = max(np.max(np.abs(a[q] - b[q])) for q in g)
        s = max(np.max(np.abs(b[q])) for q in g)
        assert d <= 1e-11 * s, (g, d / s)


def test_window_origins_cover_the_grid():
    import bench
    for n in (30, 31, 64, 128, 161, 200):
        o = bench.window_origins(n)
        cov = np.zeros(n, bool)
        for i0 in o:
            cov[i0:i0 + 30] = True
            assert 0 <= i0 and i0 + 30 <= max(n, 30)
        assert cov.all()
