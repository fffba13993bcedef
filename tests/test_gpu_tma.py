"""The flux sweeps' two ways of reading a tile: TMA box copies into shared
memory (the default) and loads through the cache by every thread (VH_TMA=0
at vh_create).  The arithmetic after the load is the same, so the two must
agree to the last bit or, failing that, far inside the parity tolerances;
the grids are ragged (row lengths that are not multiples of the 16-byte
alignment, tiles cut by every edge), FP64 and mixed, boost-invariant, 3+1D
and Cartesian."""
import os

import numpy as np
import pytest

from helpers import smooth_inputs
from viral_b200 import _abi as A
from viral_b200 import configs as C
from viral_b200.hydro import Config, Hydro

pytestmark = pytest.mark.gpu

GROUPS = [(0,), (1, 2, 3, 4), (5, 6, 7, 8, 9), (10, 11, 12, 13), (14, 15, 16, 17)]


def _run(cfg, f0, tau0, steps, tma):
    old = os.environ.get("VH_TMA")
    os.environ["VH_TMA"] = "1" if tma else "0"
    try:
        with Hydro(cfg) as H:
            assert H.sweep_uses_tma() == tma
            H.set_state(f0, tau0)
            H.step(steps)
            return H.get_state()
    finally:
        if old is None:
            del os.environ["VH_TMA"]
        else:
            os.environ["VH_TMA"] = old


def _case(which, precision):
    if which == "glauber_bi":
        cfg = C.glauber_config(nx=37, ny=29, boost_invariant=True, precision=precision)
        with C.make_hydro(cfg, C.glauber_inputs(cfg, b=4.0, seed=3)) as H:
            return cfg, H.get_state(), H.tau
    if which == "glauber_3d":
        cfg = C.glauber_config(nx=23, ny=19, nz=13, precision=precision)
        with C.make_hydro(cfg, C.glauber_inputs(cfg, b=4.0, seed=5)) as H:
            return cfg, H.get_state(), H.tau
    if which == "cartesian_3d":
        cfg = Config(nx=21, ny=18, nz=11, boost_invariant=False, coords=A.COORD_CARTESIAN, dx=0.1, dy=0.1, dz=0.1,
                     tau0=1.0, dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=13.899692864867510,
                     etas0=1 / (4 * np.pi), precision=precision)
        return cfg, smooth_inputs(cfg, cfg.tau0, seed=7), cfg.tau0
    raise ValueError(which)


@pytest.mark.parametrize("precision", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("which", ["glauber_bi", "glauber_3d", "cartesian_3d"])
def test_tma_tiles_match_cached_loads(which, precision):
    cfg, f0, tau0 = _case(which, precision)
    a = _run(cfg, f0, tau0, 12, True)
    b = _run(cfg, f0, tau0, 12, False)
    worst = 0.0
    for grp in GROUPS:
        scale = max(float(np.max(np.abs(b[q]))) for q in grp) or 1.0
        for q in grp:
            worst = max(worst, float(np.max(np.abs(a[q] - b[q]))) / scale)
    print(f"{which} precision {precision}: bitwise identical {np.array_equal(a, b)}, worst {worst:.2e}")
    assert worst <= (1e-13 if precision == A.PREC_FP64 else 1e-6)
