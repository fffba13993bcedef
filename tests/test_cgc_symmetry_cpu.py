"""Host-side properties of the optical-Glauber CGC tensor (vh_profile_cgc):
the symmetries of two equal nuclei placed at x = +/- x_pos, tracelessness of
the field tensor, the eta profile, and argument checks.  No GPU needed."""
import numpy as np

from viral_b200 import _abi as A
from viral_b200.hydro import profile_cgc

IDX = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]


def grid(T, nx, ny, gz=1):
    return T.reshape(10, gz, ny + 6, nx + 6)


def test_symmetries_and_trace():
    nx = ny = 40
    tau = 0.3
    T = grid(profile_cgc(nx, ny, 1, True, 0.1, 0.1, 0.1, tau, e_peak=500.0), nx, ny)[:, 0]
    # x -> -x: ghost-inclusive grids of even nx have x_i = -2 + (i - 3) 0.1, so
    # mirror pairs are i <-> 2*(3 + nx/2) - i; compare the interior block
    i0 = 3 + nx // 2
    sl = slice(i0 - 15, i0 + 16)
    mir = slice(i0 + 15, i0 - 16, -1)
    # x -> -x exchanges the nuclei: T^{tx} and, with beta = mu1 grad mu2 -
    # mu2 grad mu1, T^{t eta} and T^{y eta} are odd
    sx = {1: -1, 3: -1, 8: -1}
    for q in range(10):
        a, b = T[q][:, sl], T[q][:, mir]
        assert np.max(np.abs(a - sx.get(q, 1) * b)) <= 1e-11 * np.abs(T[q]).max(), q
    # y -> -y: T^{ty} and T^{y eta} are odd
    j0 = 3 + ny // 2
    sy = {2: -1, 8: -1}
    for q in range(10):
        a, b = T[q][slice(j0 - 15, j0 + 16), :], T[q][slice(j0 + 15, j0 - 16, -1), :]
        assert np.max(np.abs(a - sy.get(q, 1) * b)) <= 1e-11 * np.abs(T[q]).max(), q
    # the field tensor is traceless: T^tt - T^xx - T^yy - tau^2 T^{eta eta} = 0
    tr = T[0] - T[4] - T[7] - tau * tau * T[9]
    assert np.max(np.abs(tr)) <= 1e-12 * np.max(np.abs(T[0]))
    # T^{xy} vanishes, T^{xx} = T^{yy}; the peak e sits at the centre
    assert np.all(T[5] == 0) and np.array_equal(T[4], T[7])


def test_eta_profile():
    nx = ny = 12
    nz = 61
    T = grid(profile_cgc(nx, ny, nz, False, 0.1, 0.1, 0.1, 0.2, e_peak=100.0), nx, ny, nz + 6)
    eta = -3.0 + (np.arange(nz + 6) - 3) * 0.1
    ref = T[:, 33]  # eta = 0
    for k, h in enumerate(eta):
        a = abs(h) - 2.0
        cut = np.exp(-a * a / 2) if a >= 0 else 1.0
        assert np.allclose(T[:, k], cut * ref, rtol=1e-13, atol=0), k


def test_arguments():
    out = np.zeros((10, 16 * 16))
    L = A.lib()
    bad = [(0, 10, 0.1, 1.0), (10, 10, -0.1, 1.0), (10, 10, 0.1, 0.0)]
    for nx, ny, dx, tau in bad:
        assert L.vh_profile_cgc(nx, ny, 1, 1, dx, 0.1, 0.1, tau, 3.0, 197.0, 0.546, 12.2546, 10.0, 4.0, 100.0,
                                A.ptr(out)) == A.E_ARG
