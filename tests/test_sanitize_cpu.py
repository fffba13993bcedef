"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer: the
library's host-only sources (input generators, freeze-out surfaces and
spectra) and the oracle, built with -fsanitize=address,undefined into
_build/sanitize/ and exercised in a child Python process that preloads the
ASan runtime.  Any invalid access, overflow or undefined operation aborts the
child with the sanitizer's report.  The device code has no counterpart here
(compute-sanitizer is not used); its host-side arithmetic is shared with the
code checked here where it can be (vh_freezeout.cuh)."""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "_build", "sanitize")
FLAGS = ["-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
         "-fPIC", "-shared"]


def _runtime():
    try:
        p = subprocess.run(["g++", "-print-file-name=libasan.so"], capture_output=True, text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    path = p.stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


CHILD = textwrap.dedent("""
    import ctypes, math, sys
    ROOT, HOST, ORACLE = sys.argv[1:4]
    sys.path[:0] = [ROOT, ROOT + "/oracle", ROOT + "/tests"]
    import numpy as np
    from viral_b200 import _abi as A
    lib = ctypes.CDLL(HOST)
    for name, res, args in A.SIGNATURES:
        f = getattr(lib, name, None)
        if f is not None:
            f.restype, f.argtypes = res, args
    A.lib = lambda: lib
    import pyoracle
    _load = pyoracle._load
    pyoracle._load = lambda p: _load(ORACLE if p.endswith("liboracle.so") else p)
    from viral_b200 import configs as C
    from viral_b200 import hydro as H
    from helpers import oracle_from_inputs

    # input generators
    tab = H.eos_table_synthetic()
    assert tab.shape == (4, 2000) and np.all(np.isfinite(tab))
    e, ux, uy, pu = H.profile_gubser(17, 15, 0.1, 0.1)
    ec, uxc, uyc, pi5, puc = H.profile_gubser_cold(17, 15, 0.1, 0.1)
    assert np.all(np.isfinite(ec)) and np.all(np.isfinite(pi5))
    for bi in (True, False):
        cfg = C.glauber_config(nx=16, ny=14, nz=6, boost_invariant=bi)
        inp = C.glauber_inputs(cfg, b=5.0, seed=2)
        O = oracle_from_inputs(cfg, inp)
        tau = cfg.tau0
        for _ in range(3):
            assert O.step(tau, cfg.dtau) == 0
            tau += cfg.dtau
        assert np.all(np.isfinite(O.get_state()))
    for kw in (dict(), dict(recon=A.RECON_MINMOD)):
        cfg = C.gubser_config(nx=17, ny=17, **kw)
        O = oracle_from_inputs(cfg, C.gubser_inputs(cfg))
        assert O.step(cfg.tau0, cfg.dtau) == 0

    # freeze-out surfaces and spectra, including every cut pattern and
    # corners exactly on the isotherm
    rng = np.random.default_rng(5)
    n2 = 17 * 15
    T0 = 0.15 + 0.04 * rng.standard_normal(n2)
    T1 = 0.15 + 0.04 * rng.standard_normal(n2)
    T0[::7] = 0.15
    u = np.vstack([np.ones(n2), np.zeros((2, n2))])
    el = H.freezeout_2d(11, 9, 0.1, 0.1, 1.0, 1.1, T0, T1, u, u, 0.15)
    sp = H.cooper_frye_2d(el, 0.15, 0.14, 1.0, [0.0, 0.5, 60.0], [0.0, 1.0])
    n3 = 11 * 10 * 9
    T0 = 0.15 + 0.04 * rng.standard_normal(n3)
    T1 = 0.15 + 0.04 * rng.standard_normal(n3)
    u = np.vstack([np.ones(n3), np.zeros((3, n3))])
    el3 = H.freezeout_3d(5, 4, 3, 0.1, 0.1, 0.1, 1.0, 1.1, T0, T1, u, u, 0.15)
    sp3 = H.cooper_frye_3d(el3, 0.15, 0.14, 1.0, 0.3, [0.0, 0.5], [0.0, 1.0])
    assert len(el) > 0 and len(el3) > 0 and np.all(np.isfinite(sp)) and np.all(np.isfinite(sp3))
    # a capacity smaller than the surface: only the first rows are written
    out = np.zeros((3, 9))
    cnt = ctypes.c_longlong()
    rc = lib.vh_freezeout_2d(11, 9, 0.1, 0.1, 1.0, 1.1, A.ptr(np.ascontiguousarray(T0[:n2])),
                             A.ptr(np.ascontiguousarray(T1[:n2])), A.ptr(np.ascontiguousarray(u[:3, :n2])),
                             A.ptr(np.ascontiguousarray(u[:3, :n2])), 0.15, A.ptr(out), 3, ctypes.byref(cnt))
    assert rc == A.E_ARG and cnt.value > 3
    print("sanitized run ok")
""")


@pytest.mark.skipif(_runtime() is None, reason="g++ has no AddressSanitizer runtime")
def test_host_code_under_address_and_ub_sanitizers():
    os.makedirs(OUT, exist_ok=True)
    csrc = os.path.join(ROOT, "viral_b200", "csrc")
    host = os.path.join(OUT, "libvh_host_asan.so")
    oracle = os.path.join(OUT, "liboracle_asan.so")
    subprocess.run(["g++", "-std=c++17", *FLAGS, "-I", os.path.join(ROOT, "include"), "-I", csrc,
                    os.path.join(csrc, "vh_inputs.cpp"), os.path.join(csrc, "vh_freezeout.cpp"), "-o", host],
                   check=True, capture_output=True)
    subprocess.run(["gcc", "-std=c11", *FLAGS, "-ffp-contract=off", os.path.join(ROOT, "oracle", "oracle.c"), "-lm",
                    "-o", oracle], check=True, capture_output=True)
    env = dict(os.environ, LD_PRELOAD=_runtime(), ASAN_OPTIONS="detect_leaks=0:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, host, oracle], env=env, capture_output=True, text=True,
                       timeout=600)
    report = p.stdout[-3000:] + p.stderr[-6000:]
    assert p.returncode == 0 and "sanitized run ok" in p.stdout, report
    assert "AddressSanitizer" not in p.stderr and "runtime error" not in p.stderr, report
