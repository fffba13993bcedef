"""Generate the golden fixtures of the viscous KT step from the reference's
own code (its NEWEST5 / TXYZ5 headers compiled by oracle/Makefile into
oracle/_ref/).  Runs only where the reference tree is present:

    make -C oracle ref && python tests/golden/make_golden.py [scenario ...]

For each compile-time scenario of the reference a seeded smooth viscous
state is built on the reference's grid (pyoracle.smooth_state, then
T^{tau mu} from the oracle's closure), and the reference computes:
  * the stage-1 terms: sources, flux divergence, velocity gradients;
  * the state after two TVDRK2 steps;
  * (Milne) the Navier-Stokes initialisation of pi and T^{tau mu};
  * residuals and Jacobian of the conserved-to-primitive system at random
    points.
Outputs are stored at a seeded sample of interior cells (plus per-field
sums over the whole grid), so that the fixtures stay small.  A fifth
fixture, cart_3d_shock, is the reference's own Cartesian scenario (the
shock tube of its default TXYZ5 block) after 20 steps; a sixth, ns10_lbi,
is NEWEST10's ten-component Navier-Stokes shear tensor (CalcNS); a
seventh, bjorken, is the reference's Bjorken scenario run to tau = 10; an
eighth, cgc, the reference's Glasma initialisation (ginit.h) on one rank's
window; a ninth, gubser_is_table, cells of the reference's shipped viscous
Gubser initial table (NEWEST5/init/tempbin-8.7z).  The CPU tests
rebuild the same inputs and check the oracle against these numbers.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from pyoracle import Oracle, OracleConfig, RefBuild, RefGinit, RefNS10, grid_coords, smooth_state  # noqa: E402

# reference scenario blocks (oracle/Makefile) and the EOS / transport they compile
SCENARIOS = {
    "milne_lbi": dict(etas0=1 / (4 * math.pi), taupi_kind=0, cartesian=False, mirror=False, tau=1.3),
    "milne_3d": dict(etas0=1 / (4 * math.pi), taupi_kind=0, cartesian=False, mirror=False, tau=1.3),
    "gubser": dict(etas0=0.2, taupi_kind=1, cartesian=False, mirror=True, tau=1.3),
    "gubser_cold": dict(etas0=0.2, taupi_kind=1, cartesian=False, mirror=True, tau=1.3, cold=True),
    "cart_3d": dict(etas0=0.01 / (4 * math.pi), taupi_kind=0, cartesian=True, mirror=False, tau=1.0),
}
TS = 0.01
SEED = 7
NSAMPLE = 400


def oracle_config(R: RefBuild, sc: dict) -> OracleConfig:
    return OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=(1 if R.boost_invariant else R.gz - 6),
                        boost_invariant=R.boost_invariant, cartesian=sc["cartesian"], dx=R.dx, dy=R.dy, dz=R.dz,
                        eos_kind=0, eos_a=R.factor, etas0=sc["etas0"], etas1=0.0, hbarc=R.gevfm,
                        taupi_kind=sc["taupi_kind"], gubser_mirror=sc["mirror"], cold_plasma=sc.get("cold", False))


def inputs(R: RefBuild, sc: dict) -> np.ndarray:
    x, y, z = R.coords()
    f = smooth_state(x, y, z, sc["tau"], TS, seed=SEED, cartesian=sc["cartesian"])
    O = Oracle(oracle_config(R, sc))
    O.set_state(f)
    O.fill_tmunu(sc["tau"])
    return O.get_state()


def interior(R: RefBuild) -> np.ndarray:
    idx = np.arange(R.n)
    i, j, k = idx % R.gx, (idx // R.gx) % R.gy, idx // (R.gx * R.gy)
    return np.where((i >= R.il) & (i < R.ir) & (j >= R.jl) & (j < R.jr) & (k >= R.kl) & (k < R.kr))[0]


def make(variant: str) -> dict:
    sc = SCENARIOS[variant]
    R = RefBuild(variant)
    f = inputs(R, sc)
    rng = np.random.default_rng(123)
    cells = np.sort(rng.choice(interior(R), size=min(NSAMPLE, len(interior(R))), replace=False))
    out = {"cells": cells, "tau": sc["tau"], "ts": TS, "seed": SEED,
           "dims": np.array([R.gx, R.gy, R.gz, int(R.boost_invariant)]),
           "consts": np.array([R.dx, R.dy, R.dz, R.factor, R.gevfm])}
    R.set_state(f)
    src, res, du = R.stage_terms(sc["tau"], TS)
    out["src"] = src[:9, cells]
    out["res"] = res[:9, cells]
    out["du"] = du[:, cells]
    R.set_state(f)
    R.step(sc["tau"], TS)
    R.step(sc["tau"] + TS, TS)
    s2 = R.get_state()
    out["step2"] = s2[:, cells]
    out["step2_sum"] = s2.sum(axis=1)
    if not sc["cartesian"]:
        R.set_state(f)
        R.ns_init(sc["tau"], TS)
        ns = R.get_state()
        out["ns"] = ns[5:14, cells]
        out["ns_sum"] = ns[5:14].sum(axis=1)
    # residual / Jacobian at random points near the state of sampled cells
    xs, ps, ys, Js = [], [], [], []
    for c in cells[:40]:
        x = np.array([f[0, c], f[2, c], f[3, c], f[4, c]]) * (1 + 0.01 * rng.standard_normal(4))
        prm = np.concatenate([f[10:14, c], f[5:10, c], [0.0, sc["tau"]]])
        y, J = R.residual(x, prm)
        xs.append(x); ps.append(prm); ys.append(y); Js.append(J)
    out["res_x"], out["res_p"], out["res_y"], out["res_J"] = map(np.array, (xs, ps, ys, Js))
    return out


SHOCK_STEPS = 20


def shock_tube_state(R: RefBuild) -> np.ndarray:
    """TXYZ5's default initial state (TXYZ5/init.h:151-210): e = 16 fm^-4 for
    z < 0 and 1 fm^-4 for z >= 0, at rest, pi = 0, prevu = u, T^{tau mu}
    from the closure."""
    sc = SCENARIOS["cart_3d"]
    x, y, z = R.coords()
    f = np.zeros((18, R.n))
    f[0] = np.where(z < 0, 16.0, 1.0)
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(oracle_config(R, sc))
    O.set_state(f)
    O.fill_tmunu(0.0)
    return O.get_state()


def make_shock() -> dict:
    """The reference's Cartesian shock tube (its default TXYZ5 block),
    SHOCK_STEPS steps of dt = 0.01 from t = 0."""
    R = RefBuild("cart_3d")
    f = shock_tube_state(R)
    R.set_state(f)
    t = 0.0
    for _ in range(SHOCK_STEPS):
        R.step(t, TS)
        t += TS
    s = R.get_state()
    cells = interior(R)
    return {"cells": cells, "t": t, "ts": TS, "steps": SHOCK_STEPS,
            "dims": np.array([R.gx, R.gy, R.gz, int(R.boost_invariant)]),
            "consts": np.array([R.dx, R.dy, R.dz, R.factor, R.gevfm]),
            "state": s[:14, cells], "state_sum": s.sum(axis=1)}


BJORKEN_STEPS = 940


def make_bjorken() -> dict:
    """The reference's Bjorken scenario (NEWEST5/maindef.h:195-235,
    init.h:283-340): a uniform fluid at rest in Milne coordinates with
    e = 30 GeV/fm^3 at tau = 0.6 fm/c, run BJORKEN_STEPS steps of 0.01 fm/c to
    tau = 10 (main.cpp:208-211).  Records, after every step, the centre
    cell's temperature in fm^-1 (main.cpp:146 prints it times GEVFM/1000),
    and the final state of the centre cell."""
    R = RefBuild("bjorken")
    sc = dict(etas0=0.2, taupi_kind=2, taupi_const=0.01, cartesian=False, mirror=False)
    cfg = OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=1, boost_invariant=True, cartesian=False, dx=R.dx, dy=R.dy,
                       dz=R.dz, eos_kind=0, eos_a=R.factor, etas0=sc["etas0"], etas1=0.0, hbarc=R.gevfm,
                       taupi_kind=2, taupi_const=0.01)
    f = np.zeros((18, R.n))
    f[0] = 30.0 / R.gevfm
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(0.6)
    f = O.get_state()
    R.set_state(f)
    centre = (R.gy // 2) * R.gx + R.gx // 2
    tau, temps = 0.6, []
    for _ in range(BJORKEN_STEPS):
        R.step(tau, 0.01)
        tau += 0.01
        temps.append(R.eos(R.get_state()[0, centre])[2])
    return {"tau0": 0.6, "ts": 0.01, "steps": BJORKEN_STEPS, "centre": centre,
            "dims": np.array([R.gx, R.gy, R.gz, 1]), "consts": np.array([R.dx, R.dy, R.dz, R.factor, R.gevfm]),
            "temp": np.array(temps), "final": R.get_state()[:, centre]}


CART_BJORKEN_STEPS = 100


def make_cart_bjorken() -> dict:
    """The reference's Cartesian Bjorken block (TXYZ5/maindef.h:78-108,
    init.h:221-283): e = 30 GeV/fm^3 at rest on its 10 x 10 x 41 grid of
    0.1 fm from t = 0.6, CART_BJORKEN_STEPS steps of 0.01.  In (t, x, y, z) a
    uniform fluid at rest is an equilibrium: the record is the final state of
    the centre cell and the largest change of any field anywhere."""
    R = RefBuild("cart_bjorken")
    cfg = OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=R.gz - 6, boost_invariant=False, cartesian=True, dx=R.dx,
                       dy=R.dy, dz=R.dz, eos_kind=0, eos_a=R.factor, etas0=0.2, etas1=0.0, hbarc=R.gevfm,
                       taupi_kind=2, taupi_const=0.01)
    f = np.zeros((18, R.n))
    f[0] = 30.0 / R.gevfm
    f[1] = 1.0
    f[14] = 1.0
    O = Oracle(cfg)
    O.set_state(f)
    O.fill_tmunu(0.6)
    f = O.get_state()
    R.set_state(f)
    t = 0.6
    for _ in range(CART_BJORKEN_STEPS):
        R.step(t, 0.01)
        t += 0.01
    s = R.get_state()
    centre = ((R.gz // 2) * R.gy + R.gy // 2) * R.gx + R.gx // 2
    return {"t0": 0.6, "ts": 0.01, "steps": CART_BJORKEN_STEPS, "centre": centre,
            "dims": np.array([R.gx, R.gy, R.gz, 0]), "consts": np.array([R.dx, R.dy, R.dz, R.factor, R.gevfm]),
            "initial": f[:, centre], "final": s[:, centre], "max_change": np.abs(s - f).max(axis=1)}


CGC_SAMPLE = 1000


def make_cgc() -> dict:
    """The reference's Glasma initialisation (NEWEST5/ginit.h with its GINIT
    block: s95p EOS, tau0 = 0.1 fm/c, ts = 0.002), 3+1D with 61 eta cells, on
    the window of rank (4, 4) of its 10 x 10 layout (x, y in [-3.3, 0.2] fm
    with ghosts): the state at seeded interior cells, s95p's P there, T = 0.4
    GeV's energy density, and an s95p table (e, P, dP/de, T) for the GPU."""
    R = RefGinit(4, 4)
    f, x, y, eta = R.run()
    idx = np.arange(R.n)
    i, j, k = idx % R.gx, (idx // R.gx) % R.gy, idx // (R.gx * R.gy)
    inner = np.where((i >= R.il) & (i < R.ir) & (j >= R.jl) & (j < R.jr) & (k >= R.kl) & (k < R.kr))[0]
    cells = np.sort(np.random.default_rng(321).choice(inner, size=CGC_SAMPLE, replace=False))
    te = np.geomspace(1e-2, 1e4, 2000)
    tab = np.array([R.eos(v) for v in te])
    return {"cells": cells, "dims": np.array([R.gx, R.gy, R.gz, R.il, R.ir, R.kl, R.kr]),
            "consts": np.array([R.dx, R.dy, R.dz, R.tau0, R.ts, R.x_pos, R.flat, R.gevfm]),
            "e_at_0p4gev": R.e_at_0p4gev(), "state": f[:, cells], "x": x[cells], "y": y[cells], "eta": eta[cells],
            "P": np.array([R.eos(v)[0] for v in f[0, cells]]),
            "eos_table": np.array([te, tab[:, 0], tab[:, 1], tab[:, 2]])}


NS10_TAU = 1.3
NS10_SEED = 11


def make_ns10() -> dict:
    """NEWEST10's Navier-Stokes shear tensor (CalcNS, ten components) in its
    default compile-time block, boost invariant.  The state is the seeded
    smooth state of the other fixtures (u^eta nonzero); du[l][3], which that
    build does not compute, is seeded noise, so that every term counts."""
    R = RefNS10()
    x, y, z = grid_coords(R.gx, R.gy, R.gz, R.dx, R.dy, 0.1, True)
    f = smooth_state(x, y, z, NS10_TAU, TS, seed=SEED)
    du3 = 0.1 * np.random.default_rng(NS10_SEED).standard_normal((4, R.n))
    ns, du = R.calc_ns(f, du3, NS10_TAU, TS)
    idx = np.arange(R.n)
    i, j = idx % R.gx, idx // R.gx
    inner = np.where((i >= R.il) & (i < R.ir) & (j >= R.jl) & (j < R.jr))[0]
    cells = np.sort(np.random.default_rng(123).choice(inner, size=NSAMPLE, replace=False))
    return {"cells": cells, "tau": NS10_TAU, "ts": TS, "seed": SEED,
            "dims": np.array([R.gx, R.gy, R.gz, 1]), "consts": np.array([R.dx, R.dy, R.factor]),
            "ns": ns[:, cells], "du": du[:, cells], "ns_sum": ns[:, inner].sum(axis=1)}


def make_gubser_is_table() -> dict:
    """The reference's shipped Gubser initial table, NEWEST5/init/tempbin-8.7z
    (a 7-zip archive of one LZMA stream holding tempbin-8.dat: 326 x 326 cells
    x 8 doubles, the layout initGubser reads at NEWEST5/init.h:419-459: T,
    then pi^{tau tau}, pi^{tau x}, pi^{tau y}, pi^{xx}, pi^{xy}, pi^{yy},
    tau^2 pi^{eta eta}).  The archive's own headers are parsed here (the
    signature header, then the uncompressed header: one packed stream, one
    LZMA coder with its 5 property bytes) and the stream is decoded with the
    standard library's raw LZMA1 decoder; the CRC32 of the result is checked
    against the archive's.  Kept: the cells of the positive x axis and of the
    diagonal from the centre (163, 163), and a seeded sample."""
    import lzma
    import struct
    import zlib
    from refpath import reference_root
    path = os.path.join(reference_root(), "NEWEST5", "init", "tempbin-8.7z")
    with open(path, "rb") as fh:
        d = fh.read()
    assert d[:6] == b"7z\xbc\xaf\x27\x1c"
    next_off, next_size, _ = struct.unpack("<QQI", d[12:32])
    hdr = d[32 + next_off:32 + next_off + next_size]

    def num(b, k):  # the archive's variable-length integer at offset k
        first, mask, extra = b[k], 0x80, 0
        while extra < 8 and first & mask:
            extra += 1
            mask >>= 1
        val = int.from_bytes(b[k + 1:k + 1 + extra], "little")
        if extra < 8:
            val |= (first & (mask - 1)) << (8 * extra)
        return val, k + 1 + extra

    # kHeader, kMainStreamsInfo, kPackInfo: pack position, one stream, its size
    assert hdr[0:3] == bytes([0x01, 0x04, 0x06])
    pack_pos, k = num(hdr, 3)
    nstreams, k = num(hdr, k)
    assert nstreams == 1 and hdr[k] == 0x09
    pack_size, k = num(hdr, k + 1)
    assert hdr[k] == 0x00 and hdr[k + 1] == 0x07 and hdr[k + 2] == 0x0B  # end, kUnpackInfo, kFolder
    k += 3
    nfolders, k = num(hdr, k)
    assert nfolders == 1 and hdr[k] == 0 and hdr[k + 1] == 1  # not external, one coder
    flags = hdr[k + 2]
    idlen = flags & 0x0F
    coder = hdr[k + 3:k + 3 + idlen]
    assert coder == bytes([0x03, 0x01, 0x01]) and flags & 0x20  # LZMA, with properties
    k += 3 + idlen
    nprops, k = num(hdr, k)
    props = hdr[k:k + nprops]
    k += nprops
    assert hdr[k] == 0x0C  # kCodersUnpackSize
    unpack_size, k = num(hdr, k + 1)
    # end of the unpack info, then kSubStreamsInfo: kCRC, all defined, CRC32
    assert hdr[k] == 0x00 and hdr[k + 1] == 0x08 and hdr[k + 2] == 0x0A and hdr[k + 3] == 1
    crc = struct.unpack("<I", hdr[k + 4:k + 8])[0]
    lc, rem = props[0] % 9, props[0] // 9
    lp, pb = rem % 5, rem // 5
    dict_size = int.from_bytes(props[1:5], "little")
    dec = lzma.LZMADecompressor(format=lzma.FORMAT_RAW,
                                filters=[{"id": lzma.FILTER_LZMA1, "dict_size": dict_size, "lc": lc, "lp": lp,
                                          "pb": pb}])
    raw = dec.decompress(d[32 + pack_pos:32 + pack_pos + pack_size], max_length=unpack_size)
    assert len(raw) == unpack_size and zlib.crc32(raw) == crc
    g = int(round(math.sqrt(len(raw) // 64)))
    t = np.frombuffer(raw, dtype="<f8").reshape(g, g, 8)  # [j][i][column]
    c = g // 2
    ii = list(range(c, g)) + list(range(c, g))
    jj = [c] * (g - c) + list(range(c, g))
    rng = np.random.default_rng(5)
    ii += list(rng.integers(0, g, 64))
    jj += list(rng.integers(0, g, 64))
    ii, jj = np.array(ii), np.array(jj)
    return {"i": ii, "j": jj, "values": t[jj, ii, :].copy(), "dims": np.array([g, g]),
            "note": np.array("NEWEST5/init/tempbin-8.7z: T, pi^tt, pi^tx, pi^ty, pi^xx, pi^xy, pi^yy, tau^2 pi^ee")}


def main():
    special = {"cart_3d_shock": make_shock, "ns10_lbi": make_ns10, "bjorken": make_bjorken, "cgc": make_cgc,
               "cart_bjorken": make_cart_bjorken, "gubser_is_table": make_gubser_is_table}
    which = sys.argv[1:] or list(SCENARIOS) + list(special)
    for v in which:
        d = special[v]() if v in special else make(v)
        path = os.path.join(HERE, f"ref_{v}.npz")
        np.savez_compressed(path, **d)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
