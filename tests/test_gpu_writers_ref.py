"""vh_write against the reference's own writers, byte for byte.

oracle/ref_write.cpp compiles the reference's write.h where it lies, in
compile-time blocks with one rank: NEWEST5/write.h:51-115 (WriteResultsXY,
the central eta slice) and :225-290 (WriteResults, every cell) with 12
doubles per cell in the default block (40 x 40, and 40 x 40 x 10) and in the
BULKTEST block (10 x 10 x 4 cells, FREQ = 2: every second row and column);
NEWEST10/write.h:51-170 (the 17-variable WriteResultsXY and WriteNSXY) in
its default block.  The reference's cells hold the same state as the
handle, with Temp, P and V set the way its root-find sets them (FT(En),
EOS(En), u^i/u^tau; NEWEST5/multiroot.h:428-429, 485-492); NEWEST10's ten
pi components and Navier-Stokes tensor are the handle's own
(vh_get_primitive, vh_get_ns_pi), so those two files pin the layout.  Each
file the reference writes, res/tau%2.3ffm.bin (or res/NStau%2.3ffm.bin), must
equal vh_write's in VH_WRITE_XY, FULL, XY17 and NS_XY.  VH_WRITE_FULL17 is
WriteResults's layout with the 17-variable record, which the reference does
not write; its file is checked against the two it combines.  Late: newer
than the rest of the GPU suite."""
import os

import numpy as np
import pytest

from pyoracle import RefWrite, grid_coords, smooth_state
from viral_b200 import _abi as A
from viral_b200.hydro import Config, Hydro

pytestmark = [pytest.mark.gpu, pytest.mark.late]

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
TAU = 0.75


def _need(v):
    if not os.path.exists(os.path.join(REF, f"libref_{v}.so")):
        pytest.skip("the reference's writer builds are absent (oracle/Makefile)")


def _pair(variant, seed=3):
    _need(variant)
    W = RefWrite(variant)
    cfg = Config(nx=W.nx, ny=W.ny, nz=1 if W.boost_invariant else W.nz, boost_invariant=W.boost_invariant,
                 dx=W.dx, dy=W.dy, dz=W.dz, tau0=TAU, dtau=0.01, eos_kind=A.EOS_CONFORMAL, eos_a=W.factor,
                 etas0=1 / (4 * np.pi), hbarc=0.1973)
    x, y, z = grid_coords(W.gx, W.gy, W.gz, W.dx, W.dy, W.dz, W.boost_invariant)
    f = smooth_state(x, y, z, TAU, 0.01, seed=seed)
    if W.boost_invariant:
        for q in (4, 8, 9, 17):
            f[q] = 0.0
        for q in (1, 14):
            f[q] = np.sqrt(1 + f[q + 1] ** 2 + f[q + 2] ** 2)
    return W, cfg, f


def _ours(H, layout, every, tmp):
    p = os.path.join(tmp, f"ours_{layout}_{every}.bin")
    H.write(p, layout, every)
    with open(p, "rb") as fh:
        return fh.read()


@pytest.mark.parametrize("variant,layouts", [
    ("write_lbi", [("xy", A.WRITE_XY)]),
    ("write_3d", [("xy", A.WRITE_XY), ("full", A.WRITE_FULL)]),
    ("write_freq2", [("xy", A.WRITE_XY), ("full", A.WRITE_FULL)]),
])
def test_twelve_variable_snapshots_equal_the_reference_bytes(variant, layouts, tmp_path):
    W, cfg, f = _pair(variant)
    W.set_state(f)
    with Hydro(cfg) as H:
        H.set_state(f, TAU)
        for which, layout in layouts:
            ref = W.write(which, TAU, str(tmp_path))
            ours = _ours(H, layout, W.freq, str(tmp_path))
            assert len(ref) > 0 and ours == ref, f"{variant} {which}: {len(ours)} vs {len(ref)} bytes"


def test_newest10_snapshots_equal_the_reference_bytes(tmp_path):
    W, cfg, f = _pair("write10_lbi")
    with Hydro(cfg) as H:
        H.set_state(f, TAU)
        pi10 = H.get_primitive()["pi"]
        ns = np.zeros((11, H.n))
        ns[:10] = H.get_ns_pi()
        W.set_state(f, pi10, ns)
        ref = W.write("xy", TAU, str(tmp_path))
        assert _ours(H, A.WRITE_XY17, W.freq, str(tmp_path)) == ref
        ref_ns = W.write("ns_xy", TAU, str(tmp_path))
        assert _ours(H, A.WRITE_NS_XY, W.freq, str(tmp_path)) == ref_ns
        # FULL17: WriteResults's offsets with the 17-variable record; on a
        # boost-invariant grid it is the XY17 file
        assert _ours(H, A.WRITE_FULL17, W.freq, str(tmp_path)) == ref
