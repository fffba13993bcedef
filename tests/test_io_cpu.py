"""Input readers on the CPU: the ideal driver's ASCII initial-condition
files (NEWideal/init.h:296-345) through vh_read_ideal_profile, against a
restatement of the reference's reading loop and floor."""
import os

import numpy as np
import pytest

from viral_b200 import _abi as A
from refpath import reference_root  # noqa: E402  (oracle/ is on sys.path via conftest)
from viral_b200.hydro import read_ideal_profile


def restated(eps, vx, vy, nx, ny):
    gx, gy = nx + 6, ny + 6
    e = np.zeros((gy, gx)); X = np.zeros((gy, gx)); Y = np.zeros((gy, gx))
    e[3:3 + ny, 3:3 + nx] = eps.reshape(ny, nx)
    X[3:3 + ny, 3:3 + nx] = vx.reshape(ny, nx)
    Y[3:3 + ny, 3:3 + nx] = vy.reshape(ny, nx)
    mn = 100.0
    for v in eps:  # row by row, x fastest, as the reference reads
        if v < mn and abs(v) > 1e-5:
            mn = v
    e[e < 0.01] = mn / 10
    g = 1 / np.sqrt(1 - X * X - Y * Y)
    return e.ravel(), (g * X).ravel(), (g * Y).ravel(), mn


def write(path, a, per_line):
    with open(path, "w") as fh:
        for k in range(0, len(a), per_line):
            fh.write(" ".join("%.17g" % v for v in a[k:k + per_line]) + "\n")


def test_reader_matches_the_reference_loop(tmp_path):
    rng = np.random.default_rng(4)
    nx, ny = 9, 7
    eps = rng.uniform(0, 30, nx * ny)
    eps[[3, 10, 20]] = [0.005, 1e-6, -0.2]  # below the floor, below 1e-5, negative
    vx = rng.uniform(-0.5, 0.5, nx * ny); vy = rng.uniform(-0.5, 0.5, nx * ny)
    paths = [str(tmp_path / n) for n in ("EPS001.dat", "VX001.dat", "VY001.dat")]
    for p, a, w in zip(paths, (eps, vx, vy), (9, 5, 1)):
        write(p, a, w)
    e, ux, uy, mn = read_ideal_profile(*paths, nx, ny)
    re, rux, ruy, rmn = restated(eps, vx, vy, nx, ny)
    assert mn == rmn == -0.2
    assert np.array_equal(e, re) and np.allclose(ux, rux, rtol=1e-15, atol=0) and np.allclose(uy, ruy, rtol=1e-15)


def test_reader_errors(tmp_path):
    p = str(tmp_path / "short.dat")
    write(p, np.ones(10), 10)
    with pytest.raises(A.VhError) as ex:
        read_ideal_profile(p, p, p, 4, 4)
    assert ex.value.code == A.E_ARG
    with pytest.raises(A.VhError):
        read_ideal_profile(str(tmp_path / "missing.dat"), p, p, 2, 2)


REF_INIT = os.path.join(reference_root(), "NEWideal", "init")


@pytest.mark.skipif(not os.path.isdir(REF_INIT), reason="the reference tree is not present")
def test_reads_the_reference_files():
    """the reference's own 299x299 files, where the reference tree is present"""
    paths = [os.path.join(REF_INIT, n) for n in ("EPS001.dat", "VX001.dat", "VY001.dat")]
    e, ux, uy, mn = read_ideal_profile(*paths, 299, 299)
    raw = np.loadtxt(paths[0]).ravel()
    assert raw.size == 299 * 299
    re, _, _, rmn = restated(raw, np.loadtxt(paths[1]).ravel(), np.loadtxt(paths[2]).ravel(), 299, 299)
    assert mn == rmn and np.array_equal(e, re)
    assert np.all(e >= min(mn / 10, 0.01))
