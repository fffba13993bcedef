"""Benchmark of the viscous KT step (cell-updates per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload glauber_161x161x41] [--precision fp64|mixed]

A step is one TVDRK2 time step (two RK stages) of the whole grid.  The
default workload is the 3+1D Milne event of 161x161x41 cells (dx = dy = 0.1
fm, d eta = 0.25, dtau = 0.02 fm/c from tau0 = 0.6 fm/c), MC-Glauber Pb+Pb at
b = 7 fm (seed 0), synthetic EOS table, eta/s = 0.08, FP64.  The device state
(52 arrays x 1.3 M cells, 545 MB in FP64) is larger than L2, so no flush is
needed between steps.  value = interior cells x steps / device seconds.

One process per GPU; with N > 1 every rank evolves its own replica of the
event (the step does not shard: replicas only), value is the sum over ranks
and the time the max over ranks.

--impl reference times the reference's own CPU step (its NEWEST5 headers
built in oracle/_ref, TVDRK2 on a 40x40x10 Milne grid, the compile-time grid
of its default scenario block) in one process per host core.  --ensemble N
reports events/s of a batched ensemble; its cpu_baseline is the reference's
boost-invariant step on the host cores, extrapolated to the ensemble's cell
updates.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="glauber_161x161x41")
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--precision-report", action="store_true",
                   help="run the workload to tau_end in FP64 and mixed precision; report errors and speedup")
    p.add_argument("--tau-end", type=float, default=10.0)
    p.add_argument("--ensemble", type=int, default=0,
                   help="events/s of a batched ensemble of this many boost-invariant events")
    p.add_argument("--ensemble-precision", default="mixed", choices=["fp64", "mixed"])
    p.add_argument("--ensemble-floor", type=float, default=None,
                   help="initial energy-density floor of the ensemble events in GeV/fm^3 (default: the workload's)")
    p.add_argument("--loop-per-side", type=int, default=2,
                   help="events per grid side for the looped single-event FP64 baseline")
    p.add_argument("--adjoint", action="store_true",
                   help="adjoint/forward device-time ratio of the eps_p gradient (128x128 Glauber, 330 steps)")
    p.add_argument("--checkpoint-every", type=int, default=25)
    p.add_argument("--adjoint-steps", type=int, default=0,
                   help="steps of the adjoint workload (0: its 330 steps to tau = 7.2 fm/c); small values for profiling")
    p.add_argument("--adjoint-precision", default="both", choices=["both", "fp64", "mixed"])
    p.add_argument("--adjoint-fd", type=int, default=4,
                   help="unit directions of the finite-difference check in the adjoint mode (0: none)")
    return p.parse_args()


# ---------------------------------------------------------------- reference CPU


def _ref_worker(args):
    """One process: the reference's TVDRK2 on the compile-time grid of a
    build (milne_3d: 40x40x10 cells; milne_lbi: 40x40 boost invariant) for
    about `seconds` seconds; returns (interior cells x steps, seconds)."""
    seconds, seed, variant = (*args, "milne_3d")[:3]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from pyoracle import F_PI, F_PU, F_U, Oracle, OracleConfig, RefBuild, smooth_state
    R = RefBuild(variant)
    x, y, z = R.coords()
    tau, ts = 0.6, 0.02
    f = smooth_state(x, y, z, tau, ts, seed=seed)
    if R.boost_invariant:  # no eta flow and no eta components of pi
        for q in (F_U + 3, F_PI + 3, F_PI + 4, F_PU + 3):
            f[q] = 0.0
        for q in (F_U, F_PU):
            f[q] = np.sqrt(1 + f[q + 1] ** 2 + f[q + 2] ** 2)
    O = Oracle(OracleConfig(nx=R.gx - 6, ny=R.gy - 6, nz=1 if R.boost_invariant else R.gz - 6,
                            boost_invariant=R.boost_invariant, dx=R.dx, dy=R.dy, dz=R.dz, eos_kind=0,
                            eos_a=R.factor, etas0=1 / (4 * math.pi), hbarc=R.gevfm))
    O.set_state(f)
    O.fill_tmunu(tau)
    R.set_state(O.get_state())
    cells = (R.ir - R.il) * (R.jr - R.jl) * (R.kr - R.kl)
    R.step(tau, ts)  # warm-up
    tau += ts
    n, t0 = 0, time.perf_counter()
    while True:
        R.step(tau, ts)
        tau += ts
        n += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return cells * n, dt


def cpu_reference(seconds: float, procs: int, variant: str = "milne_3d"):
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(seconds, s, variant) for s in range(procs)])
    rate = sum(c / t for c, t in res)
    return rate, procs


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_procs() -> int:
    n = os.cpu_count() or 1
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    return max(1, min(n, 64))


# ---------------------------------------------------------------- clocks


class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for line in (self.out or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                               parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- workload


def build_workload(name: str, precision: str):
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    prec = A.PREC_MIXED if precision == "mixed" else A.PREC_FP64
    if name.startswith("glauber_"):
        nx, ny, nz = (int(v) for v in name.split("_", 1)[1].split("x"))
        cfg = C.glauber_config(nx=nx, ny=ny, nz=nz, boost_invariant=nz == 1, precision=prec)
        inp = C.glauber_inputs(cfg, b=7.0, seed=0)
        desc = {"workload": name, "grid": [nx, ny, nz], "coords": "milne", "dx_fm": 0.1,
                "deta": 0.25, "dtau_fm": 0.02, "tau0_fm": 0.6, "eos": "synthetic table (2000 rows)",
                "eta_over_s": 0.08, "ic": "MC-Glauber Pb+Pb b=7 fm seed 0, 208 nucleons, sigma_nn=6.4 fm^2",
                "recon": "WENO5", "precision": precision}
    elif name == "gubser_129":
        cfg = C.gubser_config(precision=prec)
        inp = C.gubser_inputs(cfg)
        desc = {"workload": "gubser_129", "grid": [129, 129, 1], "coords": "milne (boost invariant)",
                "dx_fm": 0.1, "dtau_fm": 0.01, "tau0_fm": 1.0, "eos": "conformal", "eta_over_s": 0.2,
                "recon": "WENO5", "precision": precision}
    else:
        raise SystemExit(f"unknown workload {name}")
    return cfg, inp, desc


def max_over_ranks(ms: float, dist, device: str) -> float:
    """The slowest rank's device time (every rank calls this)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def whole_job_rate(cells: int, steps: int, world: int, ms: float) -> float:
    """Cell updates per second of all replicas together (weak scaling)."""
    return cells * steps * world / (ms / 1e3)


def algorithmic_bytes(cfg, kernel: str) -> float:
    """Bytes one launch of `kernel` must move per interior cell (state words
    it has to read and write once; halo re-reads not counted)."""
    w = 4 if cfg.precision == 1 else 8
    if kernel.startswith("k_dir"):
        # reads e, u(4), T(4), pi(5); writes (or read+writes) res(9) and du(4)
        first = kernel.endswith("x")
        return w * (14 + (9 if first else 18) + 4)
    if kernel == "k_update_stage1":
        # reads res 9, du 12, e, u 4, pu 4, A 9; writes B 9, v1t 4, e, u 4, pu 4
        return w * (9 + 12 + 1 + 4 + 4 + 9 + 9 + 4 + 1 + 4 + 4)
    # stage 2: reads res 9, du 12, e, u 4, pu 4, B 9, A 4, v1t 4; writes A 9, e, u 4
    return w * (9 + 12 + 1 + 4 + 4 + 9 + 4 + 4 + 9 + 1 + 4)


# DRAM bytes (read + write) per interior cell and launch, from one ncu capture
# of the 121x121x31 case of the bench event (profiles/step_kernels_*.md and,
# for the FP64 stage-1 update, profiles/update_kernel_*.md; the stage-2
# figures predate the current update kernel), scaled to a full launch by the
# cells processed
MEASURED_TRAFFIC_PER_CELL = {
    ("fp64", "k_dir_x"): 150.0, ("fp64", "k_dir_y"): 239.0, ("fp64", "k_dir_eta"): 261.0,
    ("fp64", "k_update_stage1"): 538.0, ("fp64", "k_update_stage2"): 651.0,
    ("mixed", "k_dir_x"): 63.0, ("mixed", "k_dir_y"): 104.0, ("mixed", "k_dir_eta"): 114.0,
    ("mixed", "k_update_stage1"): 200.0, ("mixed", "k_update_stage2"): 223.0,
}


# the bound that does hold for the step kernels: the share of peak of the
# pipe or issue rate that limits each, from the same ncu captures
# (profiles/step_kernels_*.md, profiles/update_kernel_*.md)
MEASURED_COMPUTE_BOUND = {
    ("fp64", "k_dir_x"): ("fp64 pipe", 0.719), ("fp64", "k_dir_y"): ("fp64 pipe", 0.646),
    ("fp64", "k_dir_eta"): ("fp64 pipe", 0.682), ("fp64", "k_update_stage1"): ("fp64 pipe", 0.369),
    ("fp64", "k_update_stage2"): ("fp64 pipe", 0.273),
    ("mixed", "k_dir_x"): ("fma pipe", 0.677), ("mixed", "k_dir_y"): ("fma pipe", 0.584),
    ("mixed", "k_dir_eta"): ("fma pipe", 0.632), ("mixed", "k_update_stage2"): ("issue", 0.498),
}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_ours(args, rank, world, dist):
    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    cfg, inp, desc = build_workload(args.workload, args.precision)
    H = C.make_hydro(cfg, inp)
    A.check(A.lib().vh_set_stream(H.h, ctypes_void_p(stream.cuda_stream)), H.h)
    cells = cfg.nx * cfg.ny * (1 if cfg.boost_invariant else cfg.nz)
    launches_per_step = 2 * ((2 if cfg.boost_invariant else 3) + 1)

    H.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        H.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda")
    value = whole_job_rate(cells, args.steps, world, ms)

    # per-kernel device times (outside the timed region) for the roofline
    kt = H.time_kernels(2)
    names = ["k_dir_x", "k_dir_y", "k_dir_eta", "k_update_stage1", "k_update_stage2"]
    launches = {"k_dir_x": 4, "k_dir_y": 4, "k_dir_eta": 0 if cfg.boost_invariant else 4, "k_update_stage1": 2,
                "k_update_stage2": 2}
    per_launch = {nm: (kt[q] / launches[nm] if launches[nm] else 0.0) for q, nm in enumerate(names)}
    share = {nm: kt[q] / max(sum(kt), 1e-30) for q, nm in enumerate(names)}
    top = max(names, key=lambda nm: kt[names.index(nm)])
    peak, peak_kind = measured_peaks()
    ach = algorithmic_bytes(cfg, top) * cells / (per_launch[top] / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers
    n18 = 18 * H.n
    if args.e2e_steps <= 0:
        H.close()
        return None if rank else {"metric": METRIC, "value": value, "ms_per_step": ms / args.steps,
                                  "config": desc, "kernel_ms": dict(zip(names, kt.tolist()))}
    host = torch.empty(n18, dtype=torch.float64, pin_memory=True).numpy()
    H_state = H.get_state()
    host[:] = H_state.reshape(-1)
    tau_now = H.tau
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        A.check(A.lib().vh_set_state(H.h, A.ptr(host), tau_now), H.h)
        H.step(1)
        A.check(A.lib().vh_get_state(H.h, A.ptr(host)), H.h)
        tau_now += cfg.dtau
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_value = cells * args.e2e_steps * world / (e2e_ms / 1e3)
    H.close()

    out = None
    if rank == 0:
        clocks = clk.summary()
        out = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if cfg.precision == 0 else "f32 state / f64 root-find",
            "data": "synthetic (seeded MC-Glauber initial state)",
            "config": dict(desc, interior_cells=cells, parallelism=f"replicas x{world}",
                           l2="state (52 arrays, %.0f MB) larger than the 126 MB L2; no flush" %
                              (52 * H_state.shape[1] * (8 if cfg.precision == 0 else 4) / 1e6)),
            "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": n18 * 8, "d2h_bytes_per_step": n18 * 8,
                    "what": "vh_set_state (pinned host) + vh_step(1) + vh_get_state per step"},
            "roofline": {"bound": "hbm", "kernel": top, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_source": peak_kind,
                         "traffic": (MEASURED_TRAFFIC_PER_CELL[(args.precision, top)] * cells
                                     if (args.precision, top) in MEASURED_TRAFFIC_PER_CELL else None),
                         "algorithmic_bytes_per_cell": algorithmic_bytes(cfg, top),
                         "compute_bound_ncu": (dict(zip(("limit", "active_frac_of_peak"),
                                                        MEASURED_COMPUTE_BOUND[(args.precision, top)]))
                                               if (args.precision, top) in MEASURED_COMPUTE_BOUND else None),
                         "kernel_ms_per_launch": per_launch, "kernel_share": share},
        }
    return out


def precision_report(args):
    """Both precisions from the same initial state to tau_end: max and L2
    relative errors of e, u^mu, pi^{mu nu} of the mixed step against the FP64
    step over the interior, and the device-time ratio."""
    import numpy as np
    import torch
    from viral_b200 import configs as C
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    res = {}
    states = {}
    for prec in ("fp64", "mixed"):
        cfg, inp, desc = build_workload(args.workload, prec)
        nsteps = C.steps_between(cfg.tau0, args.tau_end, cfg.dtau)
        H = C.make_hydro(cfg, inp)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        H.step(nsteps)
        e1.record()
        torch.cuda.synchronize()
        res[prec] = {"ms": e0.elapsed_time(e1), "steps": nsteps, "tau": H.tau, "tmax_gev": H.max_temperature()}
        states[prec] = H.get_state()
        H.close()
    gx, gy, gz = cfg.gdims()
    idx = np.arange(gx * gy * gz)
    i, j, k = idx % gx, (idx // gx) % gy, idx // (gx * gy)
    kl, kr = (0, 1) if cfg.boost_invariant else (3, 3 + cfg.nz)
    m = (i >= 3) & (i < 3 + cfg.nx) & (j >= 3) & (j < 3 + cfg.ny) & (k >= kl) & (k < kr)
    a, b = states["mixed"][:, m], states["fp64"][:, m]
    groups = {"e": [0], "u": [1, 2, 3, 4], "pi": [5, 6, 7, 8, 9]}
    err = {}
    for g, qs in groups.items():
        d = a[qs] - b[qs]
        scale = np.max(np.abs(b[qs]))
        err[g] = {"max_rel": float(np.max(np.abs(d)) / scale),
                  "l2_rel": float(np.sqrt(np.sum(d * d)) / np.sqrt(np.sum(b[qs] * b[qs])))}
    out = {"report": "mixed vs fp64", "workload": args.workload, "tau_end": res["fp64"]["tau"],
           "steps": res["fp64"]["steps"], "ms_fp64": res["fp64"]["ms"], "ms_mixed": res["mixed"]["ms"],
           "speedup": res["fp64"]["ms"] / res["mixed"]["ms"], "errors": err,
           "tmax_gev": {"fp64": res["fp64"]["tmax_gev"], "mixed": res["mixed"]["tmax_gev"]},
           "error_norms": "max_rel = max|mixed-fp64| / max|fp64| over the group's components; "
                          "l2_rel = ||mixed-fp64||_2 / ||fp64||_2"}
    print(json.dumps(out), flush=True)


def ensemble(args):
    """Batched ensemble of boost-invariant MC-Glauber events (grid side drawn
    from {64,96,128,160,200}, dx = 0.1 fm, b uniform in [0,12] fm, seeds
    0..N-1, dtau = 0.02 fm/c from tau0 = 0.6 fm/c, mixed precision), each
    stopping when its maximum temperature falls below 0.15 GeV or at
    tau = 15 fm/c; one persistent kernel under a CUDA graph with the tuned
    variant.  Compared with looping the single-event FP64 step (one event at
    a time, maximum temperature read after every step as the reference's
    main loop does) on a stratified sample, extrapolated per grid side."""
    import tempfile

    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    from viral_b200.batch import Batch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    n = args.ensemble
    rng = np.random.default_rng(0)
    sides_all = np.array([64, 96, 128, 160, 200])
    sides = rng.choice(sides_all, size=n)
    bimp = rng.uniform(0.0, 12.0, size=n)
    tau0, dtau, tau_max, t_fo = 0.6, 0.02, 15.0, 0.15
    max_steps = C.steps_between(tau0, tau_max, dtau)
    prec = A.PREC_MIXED if args.ensemble_precision == "mixed" else A.PREC_FP64
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True, precision=prec)
    t_init = time.perf_counter()
    B = Batch(cfg, sides, tau0=tau0, dtau=dtau, tau_max=tau_max, t_freeze_gev=t_fo)
    floor = C.ENSEMBLE_FLOOR_GEV if args.ensemble_floor is None else args.ensemble_floor
    npart = B.init_glauber(seeds=np.arange(n), bimp=bimp, efloor_gev=floor)
    t_init = time.perf_counter() - t_init
    _, ecc2_initial = B.observables()
    cache = os.path.join(tempfile.gettempdir(), "vh_batch_tuning.txt")
    tune_ms = B.autotune(cache, probe_steps=16)
    tuning = B.tuning()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        sec, graph = B.run(max_steps)
    tau, nst, st = B.events()
    eps_p_final, _ = B.observables()
    B.close()
    okev = st != 3
    observables = {"eps2_initial_mean": float(np.mean(ecc2_initial)),
                   "eps_p_final_mean": float(np.mean(eps_p_final[okev])),
                   "corr_eps2_eps_p": float(np.corrcoef(ecc2_initial[okev], eps_p_final[okev])[0, 1]),
                   "what": "eccentricity of the initial energy density and momentum anisotropy where each event "
                           "stopped (failed events excluded), vh_batch_observables"}
    cells = (sides.astype(np.int64) ** 2)
    batch_events_s = n / sec
    batch_cells_s = float(np.sum(cells * nst)) / sec
    # looped single-event FP64 baseline on a stratified sample
    per_side = {}
    for side in (sides_all if args.loop_per_side > 0 else []):
        ts = []
        for q in range(args.loop_per_side):
            ev = int(np.where(sides == side)[0][q]) if np.sum(sides == side) > q else q
            c = C.glauber_config(nx=int(side), ny=int(side), boost_invariant=True)
            inp = C.glauber_inputs(c, b=float(bimp[ev]), seed=ev, efloor_gev=floor)
            H = C.make_hydro(c, inp)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(max_steps):
                H.step(1)
                if H.max_temperature() < t_fo or H.tau >= tau_max - 1e-9:
                    break
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            H.close()
        per_side[int(side)] = float(np.mean(ts))
    loop_seconds = float(sum(per_side[int(s_)] for s_ in sides)) if per_side else float("nan")
    out = {"metric": "events/s", "value": batch_events_s, "unit": "events/s", "n_events": n,
           "batch_seconds": sec, "cell_updates_per_s": batch_cells_s, "graph": graph, "tuning": tuning,
           "autotune_ms_per_step": tune_ms, "init_seconds": t_init,
           "steps": {"mean": float(np.mean(nst)), "min": int(nst.min()), "max": int(nst.max())},
           "stopped": {"frozen_out": int(np.sum(st == 1)), "tau_max": int(np.sum(st == 2)),
                       "failed": int(np.sum(st == 3)), "running": int(np.sum(st == 0))},
           "npart_mean": float(np.mean(npart)), "observables": observables,
           "failed_events": [{"event": int(e), "side": int(sides[e]), "b": round(float(bimp[e]), 3),
                              "steps": int(nst[e])} for e in np.where(st == 3)[0][:64]],
           "loop_fp64": {"events_per_s": n / loop_seconds, "seconds_per_event_by_side": per_side,
                         "sample": f"{args.loop_per_side} events per side, extrapolated by the side counts"},
           "speedup_vs_loop_fp64": loop_seconds / sec, "clocks": clk.summary(),
           "cpu_baseline": ensemble_cpu_baseline(args.cpu_seconds, float(np.sum(cells * nst)), n),
           "config": {"workload": "glauber ensemble", "sides": [64, 96, 128, 160, 200], "dx_fm": 0.1,
                      "b_fm": [0, 12], "dtau_fm": dtau, "tau0_fm": tau0, "tau_max_fm": tau_max,
                      "t_freeze_gev": t_fo, "floor_gev_fm3": floor,
                      "precision": f"{args.ensemble_precision} (batch) / fp64 (loop)"}}
    print(json.dumps(out), flush=True)


def ensemble_cpu_baseline(seconds: float, cell_steps: float, n_events: int) -> dict | None:
    """events/s of the reference's CPU step on the host cores for an ensemble
    of n_events that takes cell_steps interior cell updates in all: the
    reference's 2+1D TVDRK2 (its boost-invariant build, 40x40 cells) timed in
    one process per core for `seconds`, its aggregate cell-updates/s taken as
    the rate of the ensemble's events (the step's cost per cell does not
    depend on the grid side)"""
    if seconds <= 0:
        return None
    procs = reference_procs()
    rate, cores = cpu_reference(seconds, procs, "milne_lbi")
    return {"value": n_events * rate / cell_steps, "unit": "events/s", "cores": cores, "kind": "reference",
            "cell_updates_per_s": rate,
            "sample": f"{cores} processes x reference TVDRK2 (NEWEST5 headers, boost invariant, 1 MPI rank each) on "
                      f"40x40 cells for {seconds:.0f} s, extrapolated to the ensemble's {cell_steps:.4g} cell "
                      f"updates; {cpu_model()}"}


def adjoint_ratio(args):
    """Discrete adjoint of the momentum anisotropy eps_p at tau = 7.2 fm/c of
    the boost-invariant 128x128 MC-Glauber event (dx = 0.1 fm, b = 7 fm, seed
    0, floor 0.5 GeV/fm^3; 330 steps of 0.02 fm/c from 0.6 fm/c; eta/s =
    0.08 + 1.0 GeV^-1 max(T - 0.154 GeV, 0)), checkpoints every 25 steps, in
    FP64 and mixed precision.  The forward is vh_step(330) + vh_eps_p; the
    adjoint is one vh_adjoint_eps_p call (forward with checkpoints, segment
    recomputation, reverse steps, gradient export).  Device time from CUDA
    events on the handle's stream, median of --steps repetitions after
    --warmup.  The FP64 gradient is also checked against central differences
    of the FP64 forward (h = 1e-6) along 4 seeded unit directions in e0 and
    relative perturbations of (c0, c1)."""
    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    nsteps = args.adjoint_steps if args.adjoint_steps > 0 else C.ADJOINT_STEPS
    res = {}
    with ClockSampler(dev) as clk:
        modes = [("fp64", A.PREC_FP64), ("mixed", A.PREC_MIXED)]
        modes = [m_ for m_ in modes if args.adjoint_precision in ("both", m_[0])]
        for name, prec in modes:
            cfg = C.adjoint_config(128, prec)
            inp = C.adjoint_inputs(cfg)
            H = C.make_hydro(cfg, inp)
            A.check(A.lib().vh_set_stream(H.h, ctypes_void_p(stream.cuda_stream)), H.h)

            def reinit():
                H.init_profile(inp["tau"], inp["e"], inp["ux"], inp["uy"], inp["ueta"], inp["prevu"],
                               inp["pi_mode"])
                torch.cuda.synchronize()

            def timed(fn):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                out = fn()
                e1.record(stream)
                torch.cuda.synchronize()
                return e0.elapsed_time(e1), out

            fwd, adj = [], []
            for rep in range(args.warmup + args.steps):
                reinit()
                tf, eps_f = timed(lambda: (H.step(nsteps), H.eps_p())[1])
                reinit()
                ta, out = timed(lambda: H.adjoint_eps_p(nsteps, args.checkpoint_every, want_state=False))
                if rep >= args.warmup:
                    fwd.append(tf)
                    adj.append(ta)
            phases = H.adjoint_phase_times()
            res[name] = {"forward_ms": statistics.median(fwd), "adjoint_ms": statistics.median(adj),
                         "ratio": statistics.median(adj) / statistics.median(fwd), "eps_p": out[0],
                         "adjoint_phases_ms": {"forward_with_checkpoints": phases[0], "recompute_with_records": phases[1],
                                               "reverse": phases[2], "rest": phases[3]},
                         "eps_p_forward": eps_f, "grad_etas": out[3].tolist(),
                         "grad_e0_norm": float(np.linalg.norm(out[2]))}
            if name == "fp64" and args.adjoint_fd > 0:
                ge, gc = out[2], out[3]

                def eps_of(e0, c):
                    cfg2 = C.adjoint_config(128, prec, c[0], c[1])
                    with C.make_hydro(cfg2, dict(inp, e=e0)) as H2:
                        H2.step(nsteps)
                        return H2.eps_p()

                g = 134
                m = np.zeros((g, g), bool)
                m[3:131, 3:131] = True
                m = m.reshape(-1)
                rng = np.random.default_rng(1234)
                h = 1e-6
                c = np.array([0.08, 1.0])
                errs = []
                for _ in range(args.adjoint_fd):
                    v = rng.normal(size=128 * 128)
                    d = np.zeros_like(inp["e"])
                    d[m] = v / np.linalg.norm(v)
                    fd = (eps_of(inp["e"] + h * d, c) - eps_of(inp["e"] - h * d, c)) / (2 * h)
                    errs.append(abs(float(np.dot(ge, d)) - fd) / abs(fd))
                cerr = []
                for k in range(2):
                    cp = c.copy(); cm = c.copy()
                    cp[k] *= 1 + h; cm[k] *= 1 - h
                    fd = (eps_of(inp["e"], cp) - eps_of(inp["e"], cm)) / (2 * h * c[k])
                    cerr.append(abs(gc[k] - fd) / abs(fd))
                res[name]["fd_check"] = {"h": h, "e0_unit_directions_rel_err": errs, "c0_c1_rel_err": cerr}
            H.close()
    first = "fp64" if "fp64" in res else "mixed"
    out = {"metric": "adjoint/forward time ratio", "value": res[first]["ratio"], "unit": "x",
           "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "dtype": "f64" if first == "fp64" else "f32 (FP64 implicit-function solve)",
           "data": "synthetic (seeded MC-Glauber initial state)", "vs_baseline": None,
           "mixed_ratio": res["mixed"]["ratio"] if "mixed" in res else None, "detail": res, "clocks": clk.summary(),
           "config": {"workload": "glauber_128x128 adjoint", "grid": [128, 128, 1], "b_fm": 7.0, "seed": 0,
                      "floor_gev_fm3": C.ADJOINT_FLOOR_GEV, "steps": nsteps, "tau_fm": [0.6, 0.6 + 0.02 * nsteps],
                      "eta_over_s": "0.08 + 1.0 max(T - 0.154, 0)", "checkpoint_every": args.checkpoint_every,
                      "observable": "eps_p"}}
    print(json.dumps(out), flush=True)


def ctypes_void_p(v):
    import ctypes
    return ctypes.c_void_p(v)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.precision_report:
        if rank == 0:
            precision_report(args)
        return
    if args.ensemble:
        if rank == 0:
            ensemble(args)
        return
    if args.adjoint:
        if rank == 0:
            adjoint_ratio(args)
        return
    if args.impl == "reference":
        if rank != 0:
            return
        t0 = time.perf_counter()
        procs = reference_procs()
        rates = []
        for s in range(args.warmup + args.steps):
            r, _ = cpu_reference(max(1.0, args.cpu_seconds / max(1, args.steps + args.warmup)), procs)
            if s >= args.warmup:
                rates.append(r)
        value = statistics.mean(rates)
        out = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded smooth viscous state)",
               "config": {"workload": args.workload, "sample": "reference TVDRK2 on its compile-time 40x40x10 grid"},
               "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference",
                                "sample": f"{procs} processes x reference TVDRK2 (NEWEST5 headers, 1 MPI rank "
                                          f"each) on 40x40x10 cells; {cpu_model()}"},
               "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
               "wall_s": time.perf_counter() - t0}
        print(json.dumps(out), flush=True)
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    out = run_ours(args, rank, world, dist)
    if rank == 0:
        if world == 1 and args.cpu_seconds > 0 and "e2e" in out:
            procs = reference_procs()
            rate, cores = cpu_reference(args.cpu_seconds, procs)
            out["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "reference",
                                   "sample": f"{cores} processes x reference TVDRK2 (NEWEST5 headers, 1 MPI rank "
                                             f"each) on 40x40x10 cells for {args.cpu_seconds:.0f} s; {cpu_model()}"}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
