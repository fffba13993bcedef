"""INTEGRATION.md's binding run in the reference's own loop.

oracle/Makefile extracts the binding a maintainer adds to the reference (the
vh_bind.h block of INTEGRATION.md: vh_pack, vh_unpack and TVDRK2,
MaxTempGev, WriteResults[XY] over include/vh.h) and compiles it with the
reference's NEWEST5 maindef.h (default block, 40 x 40 x 10 cells) into
oracle/ref_bind_main.cpp, a program of the shape of NEWEST5/main.cpp:90-223:
cells loaded as init() leaves them, a first snapshot, then TVDRK2 / tau +=
ts / MaxTempGev / the snapshot after the first step.  After 20 steps
vh_unpack fills the cells; they must equal the oracle's 20 steps from the
same state to 1e-10, and the first snapshot must be the bytes the
reference's own WriteResults writes for that state (oracle/ref_write.cpp).
Late: newer than the rest of the GPU suite."""
import math
import os
import subprocess

import numpy as np
import pytest

from pyoracle import Oracle, OracleConfig, RefBuild, RefWrite, smooth_state
from test_gpu_parity import RUN_TOL, compare_states

pytestmark = [pytest.mark.gpu, pytest.mark.late]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "vh_bind_run_3d")
TAU0, TS, STEPS = 0.6, 0.002, 20  # TAUSTART and TS of the default block


def test_binding_in_the_reference_loop(tmp_path):
    if not (os.path.exists(BIN) and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_milne_3d.so"))):
        pytest.skip("the reference builds are absent (oracle/Makefile)")
    R = RefBuild("milne_3d")  # the same block: grid, coordinates and constants
    x, y, z = R.coords()
    f = smooth_state(x, y, z, TAU0, TS, seed=11)
    ocfg = OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=R.gz - 6, boost_invariant=False, dx=R.dx, dy=R.dy, dz=R.dz,
                        eos_kind=0, eos_a=R.factor, etas0=1 / (4 * math.pi), hbarc=R.gevfm, taupi_kind=0)
    O = Oracle(ocfg)
    O.set_state(f)
    O.fill_tmunu(TAU0)
    f0 = O.get_state()
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    f0.tofile(src)
    os.makedirs(tmp_path / "res", exist_ok=True)
    r = subprocess.run([BIN, src, dst, str(STEPS), repr(TAU0), repr(TS)], cwd=str(tmp_path), capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.count("This is tau step no.") == STEPS
    got = np.fromfile(dst, dtype=np.float64).reshape(18, -1)
    tau = TAU0
    for _ in range(STEPS):
        assert O.step(tau, TS) == 0
        tau += TS
    worst = compare_states(got, O.get_state(), RUN_TOL, fields=range(18))
    print(f"binding, {STEPS} steps in the reference's loop: max group-relative error against the oracle {worst:.2e}")
    # the first snapshot (tau0, every cell) against the reference's own writer
    W = RefWrite("write_3d")
    W.set_state(f0)
    ref = W.write("full", TAU0, str(tmp_path / "refw"))
    with open(tmp_path / "res" / ("tau%2.3ffm.bin" % TAU0), "rb") as fh:
        assert fh.read() == ref
