"""The freeze-out surface and Cooper-Frye spectra on the GPU
(vh_freezeout_{2d,3d}_device, vh_cooper_frye_{2d,3d}_device) against the
host functions on the same slices: the same element count and order, the
values to rounding (the device contracts products into FMAs), the capacity
contract, and the spectra summed per bin on the device.  Marked late: these
device paths are newer than the rest of the GPU suite."""
import ctypes

import numpy as np
import pytest
import torch

from test_freezeout_cpu import grid3
from test_freezeout_device_algo_cpu import fields_2d
from viral_b200 import _abi as A
from viral_b200.hydro import (cooper_frye_2d, cooper_frye_2d_device, cooper_frye_3d, cooper_frye_3d_device,
                              freezeout_2d, freezeout_2d_device, freezeout_3d, freezeout_3d_device)

pytestmark = [pytest.mark.gpu, pytest.mark.late]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def same_elements(got, want):
    """equal to rounding: relative 1e-12, or 1e-12 of the largest entry of
    the same kind (positions, normals, velocities), which covers components
    that cancel to rounding noise (e.g. dSigma_tau of a static surface)"""
    got = got.cpu().numpy()
    assert got.shape == want.shape
    if want.size == 0:
        return
    w = want.shape[1] // 3
    scale = np.repeat([np.abs(want[:, k * w:(k + 1) * w]).max() for k in range(3)], w)[None, :]
    assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want) + 1e-12 * scale)


def test_surface_2d_matches_the_host():
    nx, ny, dx, dy = 61, 47, 0.1, 0.15
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 11)
    host = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, T0, T1, u0, u1, 0.15)
    got = freezeout_2d_device(nx, ny, dx, dy, 1.0, 1.1, dev(T0), dev(T1), dev(u0), dev(u1), 0.15)
    assert len(host) > 1000
    same_elements(got, host)


def test_surface_3d_matches_the_host():
    nx, ny, nz, dx, dy, dz = 21, 18, 13, 0.1, 0.12, 0.2
    rng = np.random.default_rng(12)
    n = (nx + 6) * (ny + 6) * (nz + 6)
    T0 = 0.15 + 0.04 * rng.standard_normal(n)
    T1 = 0.15 + 0.04 * rng.standard_normal(n)
    T0[::13] = 0.15
    u0 = np.vstack([1 + rng.random(n), 0.3 * rng.standard_normal((3, n))])
    u1 = np.vstack([1 + rng.random(n), 0.3 * rng.standard_normal((3, n))])
    host = freezeout_3d(nx, ny, nz, dx, dy, dz, 0.8, 0.85, T0, T1, u0, u1, 0.15)
    got = freezeout_3d_device(nx, ny, nz, dx, dy, dz, 0.8, 0.85, dev(T0), dev(T1), dev(u0), dev(u1), 0.15)
    assert len(host) > 50000
    same_elements(got, host)


def test_static_ball_on_the_gpu():
    nx = ny = nz = 33
    d = 0.1
    x, y, z = grid3(nx, ny, nz, d, d, d)
    T = 0.3 * np.exp(-(x * x + y * y + z * z) / (2 * 0.6 ** 2))
    u = np.zeros((4, x.size))
    u[0] = 1.0
    host = freezeout_3d(nx, ny, nz, d, d, d, 1.0, 1.05, T, T, u, u, 0.15)
    got = freezeout_3d_device(nx, ny, nz, d, d, d, 1.0, 1.05, dev(T), dev(T), dev(u), dev(u), 0.15)
    same_elements(got, host)


def test_capacity_on_the_gpu():
    nx, ny, dx, dy = 31, 31, 0.1, 0.1
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 13)
    host = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, T0, T1, u0, u1, 0.15)
    cap = len(host) // 3
    out = torch.full((cap + 4, 9), 7.0, dtype=torch.float64, device="cuda")
    ts = [dev(T0), dev(T1), dev(u0), dev(u1)]
    cnt = ctypes.c_longlong()
    rc = A.lib().vh_freezeout_2d_device(nx, ny, dx, dy, 1.0, 1.1, *[t.data_ptr() for t in ts], 0.15, out.data_ptr(),
                                        cap, ctypes.byref(cnt), torch.cuda.current_stream().cuda_stream)
    assert rc == A.E_ARG and cnt.value == len(host)
    same_elements(out[:cap], host[:cap])
    assert torch.all(out[cap:] == 7.0)


def test_spectra_match_the_host():
    nx, ny, dx, dy = 41, 41, 0.2, 0.2
    T0, T1, u0, u1 = fields_2d(nx, ny, dx, dy, 14)
    el = freezeout_2d(nx, ny, dx, dy, 1.0, 1.1, np.abs(T0), np.abs(T1), u0, u1, 0.15)
    pt, phi = np.linspace(0.0, 3.0, 7), np.linspace(0, 2 * np.pi, 9, endpoint=False)
    host = cooper_frye_2d(el, 0.15, 0.7, 3.0, pt, phi)
    got = cooper_frye_2d_device(dev(el), 0.15, 0.7, 3.0, pt, phi)
    assert np.allclose(got, host, rtol=1e-11, atol=0)

    x, y, z = grid3(17, 17, 9, 0.2, 0.2, 0.3)
    T = 0.3 * np.exp(-(x * x + y * y) / 2 - z * z / 4)
    u = np.vstack([np.sqrt(1 + 0.09 * (x * x + y * y)), 0.3 * x, 0.3 * y, np.zeros_like(x)])
    el3 = freezeout_3d(17, 17, 9, 0.2, 0.2, 0.3, 1.0, 1.1, T, 0.9 * T, u, u, 0.15)
    for yy in (0.0, 0.4):
        host3 = cooper_frye_3d(el3, 0.15, 0.7, 3.0, yy, pt, phi)
        got3 = cooper_frye_3d_device(dev(el3), 0.15, 0.7, 3.0, yy, pt, phi)
        assert np.allclose(got3, host3, rtol=1e-11, atol=0)


def test_freezeout_step_follows_a_run():
    """vh_freezeout_step during a viscous Gubser run: the surface between
    consecutive steps from the handle's own slices equals the host surface
    of the same slices read back with vh_get_primitive"""
    from viral_b200 import configs as C
    cfg = C.gubser_config(nx=33, ny=33)
    with C.make_hydro(cfg, C.gubser_inputs(cfg)) as H:
        p = H.get_primitive()
        tfo = 0.85 * p["T"].max()
        assert H.freezeout_step(tfo).shape == (0, 9)  # the first call keeps the slice
        prev, total = (H.tau, p["T"], p["u"]), 0
        for _ in range(6):
            H.step(1)
            got = H.freezeout_step(tfo)
            q = H.get_primitive()
            want = freezeout_2d(cfg.nx, cfg.ny, cfg.dx, cfg.dy, prev[0], H.tau, prev[1], q["T"], prev[2], q["u"], tfo)
            same_elements(got, want)
            total += len(want)
            prev = (H.tau, q["T"], q["u"])
        assert total > 50
        with pytest.raises(A.VhError) as err:  # no step since the last slice
            H.freezeout_step(tfo)
        assert err.value.code == A.E_STATE

        # too small an output: the count comes back and the slice is kept
        H.step(1)
        q = H.get_primitive()
        want = freezeout_2d(cfg.nx, cfg.ny, cfg.dx, cfg.dy, prev[0], H.tau, prev[1], q["T"], prev[2], q["u"], tfo)
        assert len(want) > 2
        small = torch.zeros((2, 9), dtype=torch.float64, device="cuda")
        cnt = ctypes.c_longlong()
        assert A.lib().vh_freezeout_step(H.h, tfo, small.data_ptr(), 2, ctypes.byref(cnt)) == A.E_ARG
        assert cnt.value == len(want)
        same_elements(H.freezeout_step(tfo), want)
