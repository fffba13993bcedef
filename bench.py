"""Benchmark of the viscous KT step: cell-updates/s, events/s, mixed vs FP64
at stated error, adjoint/forward ratio.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload glauber_161x161x41] [--precision fp64|mixed]
                    [--sub mixed,ensemble,adjoint]

A step is one TVDRK2 time step (two RK stages) of the whole grid.  The
headline workload is the 3+1D Milne event of 161x161x41 cells (dx = dy = 0.1
fm, d eta = 0.25, dtau = 0.02 fm/c from tau0 = 0.6 fm/c), MC-Glauber Pb+Pb at
b = 7 fm (seed 0), synthetic EOS table, eta/s = 0.08, FP64.  The device state
(52 arrays x 1.3 M cells, 545 MB in FP64) is larger than L2, so no flush is
needed between steps.  value = interior cells x steps / device seconds.

At N = 1 the same JSON line also carries, each with its own CUDA-event
timing and clock record:
  mixed     the precision form of the same event (FP32 state, FP64
            root-find): ms per step, speed-up over the FP64 line, errors of
            e, u^mu, pi^{mu nu} against FP64 at steps 10, 50 and W+K;
  ensemble  2048 boost-invariant events in one persistent kernel under a CUDA
            graph (mixed and FP64), completed events/s, failed events apart,
            the looped single-event FP64 step and the reference's CPU step;
  adjoint   the eps_p gradient of the 128x128 event: adjoint/forward device
            time in FP64 and mixed, checked against central differences.

One process per GPU; with N > 1 every rank evolves its own replica of the
event (the step does not shard: replicas only), value is the sum over ranks
and the time the max over ranks; the sub-records run at N = 1 only.

--impl reference times the reference's own CPU step (its NEWEST5 headers
built in oracle/_ref, the GINIT block's EOS hooks on the synthetic table) on
30x30x41 windows cut from the same Glauber state, in one process per host
core, and prints the same config.
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
    p.add_argument("--e2e-steps", type=int, default=12)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--precision-report", action="store_true",
                   help="run the workload to tau_end in FP64 and mixed precision; report errors and speedup")
    p.add_argument("--tau-end", type=float, default=10.0)
    p.add_argument("--sub", default="mixed,ensemble,adjoint",
                   help="sub-records of the N = 1 line (comma list of mixed, ensemble, adjoint; 'none')")
    p.add_argument("--ensemble", type=int, default=0,
                   help="standalone: events/s of a batched ensemble of this many boost-invariant events")
    p.add_argument("--ensemble-events", type=int, default=2048, help="events of the ensemble sub-record")
    p.add_argument("--ensemble-fp64", type=int, default=1, help="also run the ensemble batch in FP64 (1/0)")
    p.add_argument("--ensemble-floor", type=float, default=None,
                   help="initial energy-density floor of the ensemble events in GeV/fm^3 (default: the workload's)")
    p.add_argument("--loop-per-side", type=int, default=2,
                   help="events per grid side for the looped single-event FP64 baseline")
    p.add_argument("--adjoint", action="store_true",
                   help="standalone: adjoint/forward device-time ratio of the eps_p gradient (128x128 Glauber)")
    p.add_argument("--checkpoint-every", type=int, default=25)
    p.add_argument("--adjoint-steps", type=int, default=0,
                   help="steps of the adjoint workload (0: its 330 steps to tau = 7.2 fm/c); small values for profiling")
    p.add_argument("--adjoint-reps", type=int, default=5, help="timed repetitions of forward and adjoint")
    p.add_argument("--adjoint-precision", default="both", choices=["both", "fp64", "mixed"])
    p.add_argument("--adjoint-fd", type=int, default=4,
                   help="unit directions of the finite-difference check in the adjoint mode (0: none)")
    p.add_argument("--ref-sample-seconds", type=float, default=2.0,
                   help="--impl reference: step seconds per process in one sample (one sample per step)")
    return p.parse_args()


# ---------------------------------------------------------------- reference CPU
#
# The reference's own CPU step (its NEWEST5 headers compiled in oracle/_ref)
# on windows cut from the benchmarked state.  Its grid is a compile-time
# constant: the table-EOS builds (libref_window_3d / _lbi: the GINIT scenario
# block with its EOS hooks on a run-time table) step 30 x 30 x nz cells of
# one rank, so the 161 x 161 x 41 event is cut into 6 x 6 such windows (the
# reference's own MPI decomposition, with copy boundaries where its halo
# exchange would run).  Each host process steps its share of the windows in
# turn; only the TVDRK2 calls are timed.

REF_WINDOW = 30  # interior cells per window side (XL/XS of the GINIT block)


def window_origins(n: int, w: int = REF_WINDOW) -> list:
    """ghost-inclusive origins of w-wide windows covering n interior cells
    (the last one flush with the far edge)"""
    if n <= w:
        return [0]
    o = list(range(0, n - w + 1, w))
    if o[-1] != n - w:
        o.append(n - w)
    return o


def glauber_rest_state(cfg, inp) -> "np.ndarray":
    """18-field state of a Glauber initial condition at rest with pi = 0:
    T^{tau tau} = e, T^{tau i} = 0, prevu = u = (1, 0, 0, 0)"""
    import numpy as np
    gx, gy, gz = cfg.gdims()
    n = gx * gy * gz
    f = np.zeros((18, n))
    f[0] = np.asarray(inp["e"]).reshape(n)
    f[1] = 1.0
    f[10] = f[0]
    f[14] = 1.0
    return f


def _ref_window_worker(args):
    """One process: the reference's TVDRK2 on its windows, round robin, for
    n_samples samples of about `seconds` each (at least one window step per
    sample); returns [(interior cells x steps, step seconds)] per sample."""
    variant, state_path, dims, origins, seconds, n_samples, tau0, dtau, eos_path = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from pyoracle import RefBuild
    R = RefBuild(variant)
    R.set_eos_table(np.load(eos_path))
    gx, gy, gz = dims
    F = np.load(state_path, mmap_mode="r").reshape(18, gz, gy, gx)
    wins = []
    for (i0, j0) in origins:
        f = np.ascontiguousarray(F[:, :R.gz, j0:j0 + R.gy, i0:i0 + R.gx]).reshape(18, -1)
        wins.append([f, tau0])
    cells = (R.ir - R.il) * (R.jr - R.jl) * (R.kr - R.kl)
    out, q = [], 0
    for _ in range(n_samples):
        done, t_step = 0, 0.0
        while True:
            w = wins[q % len(wins)]
            R.set_state(w[0])
            t0 = time.perf_counter()
            R.step(w[1], dtau)
            t_step += time.perf_counter() - t0
            w[0] = R.get_state()
            w[1] += dtau
            done += cells
            q += 1
            if t_step >= seconds:
                break
        out.append((done, t_step))
    return out


def reference_windows(workload: str, seconds: float, n_samples: int, procs: int):
    """Aggregate cell-updates/s of the reference's CPU step over `procs` host
    processes on windows of a Glauber state of `workload` (the benchmarked
    161x161x41 event, or a boost-invariant event of the ensemble): one rate
    per sample (sum over processes of cells / their step seconds)."""
    import tempfile

    import numpy as np
    from viral_b200 import configs as C
    if workload == "ensemble":
        cfg = C.glauber_config(nx=128, ny=128, boost_invariant=True)
        inp = C.glauber_inputs(cfg, b=7.0, seed=0, efloor_gev=C.ENSEMBLE_FLOOR_GEV)
        variant = "window_lbi"
    else:
        nx, ny, nz = (int(v) for v in workload.split("_", 1)[1].split("x"))
        if nz != 41:
            raise SystemExit("the reference's 3+1D window build has 41 eta cells")
        cfg = C.glauber_config(nx=nx, ny=ny, nz=nz)
        inp = C.glauber_inputs(cfg, b=7.0, seed=0)
        variant = "window_3d"
    f = glauber_rest_state(cfg, inp)
    gdims = cfg.gdims()
    origins = [(i0, j0) for j0 in window_origins(cfg.ny) for i0 in window_origins(cfg.nx)]
    with tempfile.TemporaryDirectory() as td:
        sp, ep = os.path.join(td, "state.npy"), os.path.join(td, "eos.npy")
        np.save(sp, f)
        np.save(ep, np.asarray(cfg.eos_table))
        procs = max(1, min(procs, len(origins)))
        jobs = [(variant, sp, gdims, origins[p::procs], seconds, n_samples, cfg.tau0, cfg.dtau, ep)
                for p in range(procs)]
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_ref_window_worker, jobs)
    rates = [sum(r[k][0] / r[k][1] for r in res) for k in range(n_samples)]
    desc = (f"{procs} processes x the reference's TVDRK2 (NEWEST5 headers, GINIT block with the synthetic EOS table, "
            f"1 MPI rank each) on {len(origins)} windows of {REF_WINDOW}x{REF_WINDOW}"
            f"{'' if cfg.boost_invariant else 'x' + str(cfg.nz)} cells cut from the "
            f"{'boost-invariant 128x128 ensemble event' if workload == 'ensemble' else workload} Glauber state "
            f"(eta/s = 1/4pi, d eta = 0.1 in that block; copy boundaries at window faces)")
    return rates, procs, desc


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
    """nvidia-smi samples (every 100 ms) around a timed region: entering waits
    for the sampler's first line, leaving waits for one more, so that even a
    region shorter than the interval is bracketed by samples taken under load."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []
        self.thread = None
        self.first = 0
        self.out = ""

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)

    def _wait_for(self, n: int, limit_s: float):
        t0 = time.time()
        while len(self.lines) < n and time.time() - t0 < limit_s and self.proc.poll() is None:
            time.sleep(0.005)

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        self._wait_for(1, 5.0)
        self.first = max(len(self.lines) - 1, 0)
        return self

    def __exit__(self, *a):
        self.out = ""
        if not self.proc:
            return
        self._wait_for(len(self.lines) + 1, 1.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self.thread.join(timeout=5)
        self.out = "".join(self.lines[self.first:])

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


def build_workload(name: str, precision: str, inputs: bool = True):
    """(Config, inputs or None, description) of a named workload"""
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    prec = A.PREC_MIXED if precision == "mixed" else A.PREC_FP64
    inp = None
    if name.startswith("glauber_"):
        nx, ny, nz = (int(v) for v in name.split("_", 1)[1].split("x"))
        cfg = C.glauber_config(nx=nx, ny=ny, nz=nz, boost_invariant=nz == 1, precision=prec)
        if inputs:
            inp = C.glauber_inputs(cfg, b=7.0, seed=0)
        desc = {"workload": name, "grid": [nx, ny, nz], "coords": "milne", "dx_fm": 0.1,
                "deta": 0.25, "dtau_fm": 0.02, "tau0_fm": 0.6, "eos": "synthetic table (2000 rows)",
                "eta_over_s": 0.08, "ic": "MC-Glauber Pb+Pb b=7 fm seed 0, 208 nucleons, sigma_nn=6.4 fm^2",
                "recon": "WENO5", "precision": precision}
    elif name == "gubser_129":
        cfg = C.gubser_config(precision=prec)
        if inputs:
            inp = C.gubser_inputs(cfg)
        desc = {"workload": "gubser_129", "grid": [129, 129, 1], "coords": "milne (boost invariant)",
                "dx_fm": 0.1, "dtau_fm": 0.01, "tau0_fm": 1.0, "eos": "conformal", "eta_over_s": 0.2,
                "recon": "WENO5", "precision": precision}
    else:
        raise SystemExit(f"unknown workload {name}")
    return cfg, inp, desc


def line_config(name: str, precision: str, world: int) -> dict:
    """the `config` of the JSON line: the same dict for both arms"""
    cfg, _, desc = build_workload(name, precision, inputs=False)
    gx, gy, gz = cfg.gdims()
    cells = cfg.nx * cfg.ny * (1 if cfg.boost_invariant else cfg.nz)
    mb = 52 * gx * gy * gz * (8 if precision == "fp64" else 4) / 1e6
    return dict(desc, interior_cells=cells, parallelism=f"replicas x{world}",
                l2="state (52 arrays, %.0f MB) larger than the 126 MB L2; no flush" % mb)


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
# of the 121x121x31 case of the bench event (profiles/step_kernels_*.md for the
# sweeps, profiles/update_kernel_*.md for the updates), scaled to a full launch
# by the cells processed
MEASURED_TRAFFIC_PER_CELL = {
    ("fp64", "k_dir_x"): 153.0, ("fp64", "k_dir_y"): 230.0, ("fp64", "k_dir_eta"): 258.0,
    ("fp64", "k_update_stage1"): 469.0, ("fp64", "k_update_stage2"): 500.0,
    ("mixed", "k_dir_x"): 65.0, ("mixed", "k_dir_y"): 104.0, ("mixed", "k_dir_eta"): 114.0,
    ("mixed", "k_update_stage1"): 192.0, ("mixed", "k_update_stage2"): 226.0,
}


# the bound that does hold for the step kernels: the share of peak of the
# pipe or issue rate that limits each, from the same ncu captures
MEASURED_COMPUTE_BOUND = {
    ("fp64", "k_dir_x"): ("fp64 pipe", 0.753), ("fp64", "k_dir_y"): ("fp64 pipe", 0.724),
    ("fp64", "k_dir_eta"): ("fp64 pipe", 0.756), ("fp64", "k_update_stage1"): ("fp64 pipe", 0.323),
    ("fp64", "k_update_stage2"): ("fp64 pipe", 0.347),
    ("mixed", "k_dir_x"): ("fma pipe", 0.680), ("mixed", "k_dir_y"): ("fma pipe", 0.650),
    ("mixed", "k_dir_eta"): ("fma pipe", 0.693), ("mixed", "k_update_stage1"): ("issue", 0.503),
    ("mixed", "k_update_stage2"): ("issue", 0.507),
}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def timed_steps(H, stream, k: int, dev: int):
    """device ms of k steps of handle H on `stream` (CUDA events), with the
    clocks sampled during them"""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        H.step(k)
        ev1.record(stream)
        torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), clk.summary()


KERNELS = ["k_dir_x", "k_dir_y", "k_dir_eta", "k_update_stage1", "k_update_stage2"]


def kernel_times(H, cfg):
    """per-launch device ms and share of each step kernel over 2 steps
    (vh_time_kernels: events around every launch, outside the timed region)"""
    kt = H.time_kernels(2)
    launches = {"k_dir_x": 4, "k_dir_y": 4, "k_dir_eta": 0 if cfg.boost_invariant else 4, "k_update_stage1": 2,
                "k_update_stage2": 2}
    per_launch = {nm: (kt[q] / launches[nm] if launches[nm] else 0.0) for q, nm in enumerate(KERNELS)}
    share = {nm: kt[q] / max(sum(kt), 1e-30) for q, nm in enumerate(KERNELS)}
    top = max(KERNELS, key=lambda nm: kt[KERNELS.index(nm)])
    return per_launch, share, top


def roofline(cfg, precision: str, cells: int, per_launch: dict, share: dict, top: str) -> dict:
    peak, peak_kind = measured_peaks()
    ach = algorithmic_bytes(cfg, top) * cells / (per_launch[top] / 1e3) / 1e9
    return {"bound": "hbm", "kernel": top, "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind,
            "traffic": (MEASURED_TRAFFIC_PER_CELL[(precision, top)] * cells
                        if (precision, top) in MEASURED_TRAFFIC_PER_CELL else None),
            "algorithmic_bytes_per_cell": algorithmic_bytes(cfg, top),
            "compute_bound_ncu": (dict(zip(("limit", "active_frac_of_peak"), MEASURED_COMPUTE_BOUND[(precision, top)]))
                                  if (precision, top) in MEASURED_COMPUTE_BOUND else None),
            "kernel_ms_per_launch": per_launch, "kernel_share": share}


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
    ms, clocks = timed_steps(H, stream, args.steps, dev)
    ms = max_over_ranks(ms, dist, "cuda")
    value = whole_job_rate(cells, args.steps, world, ms)

    per_launch, share, top = kernel_times(H, cfg)

    # end to end through the C ABI with pinned host buffers
    n18 = 18 * H.n
    if args.e2e_steps <= 0:
        H.close()
        return None if rank else {"metric": METRIC, "value": value, "ms_per_step": ms / args.steps,
                                  "config": desc, "kernel_ms_per_launch": per_launch}
    state0 = H.get_state().reshape(-1).copy()
    tau_now = H.tau
    H.close()
    e2e_ms, serial_ms = e2e_runs(cfg, state0, tau_now, args.e2e_steps, stream)
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    serial_ms = max_over_ranks(serial_ms, dist, "cuda")
    e2e_value = cells * args.e2e_steps * world / (e2e_ms / 1e3)
    e2e_serial = cells * args.e2e_steps * world / (serial_ms / 1e3)

    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if cfg.precision == 0 else "f32 state / f64 root-find",
        "data": "synthetic (seeded MC-Glauber initial state)",
        "config": line_config(args.workload, args.precision, world),
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": n18 * 8, "d2h_bytes_per_step": n18 * 8,
                "steps": args.e2e_steps, "handles": E2E_HANDLES,
                "what": ("every step: vh_set_state of the full 18-field state from pinned host memory, vh_step(1), "
                         "vh_get_state of the full state into pinned host memory; %d handles on their own CUDA "
                         "streams, each driven by its own host thread and each feeding its result back as its next "
                         "input, take the steps in turn, so one handle's copies overlap the others' (PCIe is full "
                         "duplex); device time from an event before the first call to one after the last, across "
                         "all the streams" % E2E_HANDLES),
                "serial_value": e2e_serial,
                "serial_what": "the same calls on one handle, one step after the other"},
        "roofline": roofline(cfg, args.precision, cells, per_launch, share, top),
    }


E2E_HANDLES = 3


def e2e_runs(cfg, state0, tau0, steps: int, stream, nh: int = E2E_HANDLES):
    """device milliseconds of `steps` end-to-end steps through the C ABI
    (vh_set_state from pinned host memory, vh_step(1), vh_get_state into it):
    pipelined over nh handles, each on its own stream and host thread, and
    serial on one.  Each handle's cycle is host-to-device copy, step,
    device-to-host copy; with three in flight the copy engines of both
    directions stay busy (two leave gaps)."""
    import threading
    import torch
    from viral_b200 import _abi as A
    from viral_b200.hydro import Hydro
    n18 = state0.size
    streams = [torch.cuda.Stream() for _ in range(nh)]
    hs = [Hydro(cfg) for _ in range(nh)]
    bufs = [torch.empty(n18, dtype=torch.float64, pin_memory=True).numpy() for _ in range(nh)]
    try:
        for k in range(nh):
            A.check(A.lib().vh_set_stream(hs[k].h, ctypes_void_p(streams[k].cuda_stream)), hs[k].h)
            bufs[k][:] = state0
            # one untimed round trip (the transfer buffer is allocated on first use)
            A.check(A.lib().vh_set_state(hs[k].h, A.ptr(bufs[k]), tau0), hs[k].h)
            hs[k].step(1)
            A.check(A.lib().vh_get_state(hs[k].h, A.ptr(bufs[k])), hs[k].h)
            bufs[k][:] = state0
        torch.cuda.synchronize()
        errors = []

        def drive(k, count):
            tau = tau0
            try:
                for _ in range(count):
                    A.check(A.lib().vh_set_state(hs[k].h, A.ptr(bufs[k]), tau), hs[k].h)
                    hs[k].step(1)
                    A.check(A.lib().vh_get_state(hs[k].h, A.ptr(bufs[k])), hs[k].h)
                    tau += cfg.dtau
            except Exception as ex:  # reported after the join
                errors.append(ex)

        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        for k in range(1, nh):
            streams[k].wait_event(e0)
        threads = [threading.Thread(target=drive, args=(k, steps // nh + (1 if k < steps % nh else 0)))
                   for k in range(nh)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        for k in range(1, nh):
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(streams[k])
            streams[0].wait_event(e1)
        e2 = torch.cuda.Event(enable_timing=True)
        e2.record(streams[0])
        torch.cuda.synchronize()
        pipelined = e0.elapsed_time(e2)

        # serial: one handle, the calls one after the other
        bufs[0][:] = state0
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(streams[0])
        drive(0, steps)
        s1.record(streams[0])
        torch.cuda.synchronize()
        if errors:
            raise errors[0]
        return pipelined, s0.elapsed_time(s1)
    finally:
        for hh in hs:
            hh.close()


# ---------------------------------------------------------------- mixed precision


def interior(cfg):
    import numpy as np
    gx, gy, gz = cfg.gdims()
    idx = np.arange(gx * gy * gz)
    i, j, k = idx % gx, (idx // gx) % gy, idx // (gx * gy)
    kl, kr = (0, 1) if cfg.boost_invariant else (3, 3 + cfg.nz)
    return (i >= 3) & (i < 3 + cfg.nx) & (j >= 3) & (j < 3 + cfg.ny) & (k >= kl) & (k < kr)


def state_errors(a, b, m) -> dict:
    """max and L2 relative differences of a against b over the interior mask
    m, per group: e; u^mu; pi^{mu nu}"""
    import numpy as np
    out = {}
    for g, qs in {"e": [0], "u": [1, 2, 3, 4], "pi": [5, 6, 7, 8, 9]}.items():
        x, y = a[qs][:, m], b[qs][:, m]
        d = x - y
        out[g] = {"max_rel": float(np.max(np.abs(d)) / np.max(np.abs(y))),
                  "l2_rel": float(np.sqrt(np.sum(d * d)) / np.sqrt(np.sum(y * y)))}
    return out


ERROR_NORMS = ("max_rel = max|a-b| / max|b| over the group's components and the interior cells; "
               "l2_rel = ||a-b||_2 / ||b||_2; groups e, u^mu (4), pi^{mu nu} (5 stored)")


def mixed_record(args, fp64_ms_per_step: float) -> dict:
    """The precision form on the same event: FP32 state, fluxes,
    reconstruction and sources, FP64 root-find and conservation sums.  Device
    ms per step over --steps steps after --warmup (as the FP64 line), the
    speed-up over the FP64 line, and the errors of e, u^mu, pi^{mu nu}
    against an FP64 run from the same initial state at step 10, step 50 and
    the step the timed run ended on; beside them, the same errors of an FP64
    run whose initial e was perturbed by 1e-7 (relative, seeded), the size of
    FP32 rounding: where that baseline is large the event's trajectories
    have separated, which no reduced-precision step can avoid."""
    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    dev = int(os.environ.get("LOCAL_RANK", 0))
    stream = torch.cuda.current_stream()
    cfg32, inp, desc = build_workload(args.workload, "mixed")
    cfg64, _, _ = build_workload(args.workload, "fp64", inputs=False)
    cells = cfg32.nx * cfg32.ny * (1 if cfg32.boost_invariant else cfg32.nz)
    H = C.make_hydro(cfg32, inp)
    A.check(A.lib().vh_set_stream(H.h, ctypes_void_p(stream.cuda_stream)), H.h)
    H.step(args.warmup)
    torch.cuda.synchronize()
    ms, clocks = timed_steps(H, stream, args.steps, dev)
    per_launch, share, top = kernel_times(H, cfg32)
    H.close()
    m = interior(cfg64)
    marks = sorted({10, 50, args.warmup + args.steps})
    rng = np.random.default_rng(7)
    inp_p = dict(inp, e=np.asarray(inp["e"]) * (1 + 1e-7 * rng.uniform(-1, 1, size=np.asarray(inp["e"]).shape)))
    errs, base = {}, {}
    with C.make_hydro(cfg64, inp) as H64, C.make_hydro(cfg32, inp) as H32, C.make_hydro(cfg64, inp_p) as Hp:
        done = 0
        for k in marks:
            for h in (H64, H32, Hp):
                h.step(k - done)
            done = k
            ref = H64.get_state()
            errs[str(k)] = state_errors(H32.get_state(), ref, m)
            base[str(k)] = state_errors(Hp.get_state(), ref, m)
        tau_end = H64.tau
    ms_step = ms / args.steps
    return {"metric": METRIC, "value": cells * args.steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms_step,
            "steps": args.steps, "warmup": args.warmup, "speedup_vs_fp64": fp64_ms_per_step / ms_step,
            "dtype": "f32 state, fluxes, reconstruction, sources / f64 root-find, EOS inversion, conservation sums",
            "errors_vs_fp64": errs, "fp64_perturbed_1e-7_vs_fp64": base, "error_steps": marks,
            "error_tau_end_fm": tau_end, "error_norms": ERROR_NORMS, "clocks": clocks,
            "gpu_launches": 2 * ((2 if cfg32.boost_invariant else 3) + 1) * args.steps,
            "roofline": roofline(cfg32, "mixed", cells, per_launch, share, top),
            "config": dict(desc, workload=args.workload + " (precision form)")}


def precision_report(args):
    """Both precisions from the same initial state to tau_end: max and L2
    relative errors of e, u^mu, pi^{mu nu} of the mixed step against the FP64
    step over the interior, and the device-time ratio."""
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
    err = state_errors(states["mixed"], states["fp64"], interior(cfg))
    out = {"report": "mixed vs fp64", "workload": args.workload, "tau_end": res["fp64"]["tau"],
           "steps": res["fp64"]["steps"], "ms_fp64": res["fp64"]["ms"], "ms_mixed": res["mixed"]["ms"],
           "speedup": res["fp64"]["ms"] / res["mixed"]["ms"], "errors": err,
           "tmax_gev": {"fp64": res["fp64"]["tmax_gev"], "mixed": res["mixed"]["tmax_gev"]},
           "error_norms": ERROR_NORMS}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- ensemble


def ensemble_events(n: int):
    """the ensemble's grid sides (from {64, 96, 128, 160, 200}) and impact
    parameters (uniform in [0, 12] fm), seeded"""
    import numpy as np
    rng = np.random.default_rng(0)
    sides = rng.choice(np.array([64, 96, 128, 160, 200]), size=n)
    bimp = rng.uniform(0.0, 12.0, size=n)
    return sides, bimp


ENS_TAU0, ENS_DTAU, ENS_TAU_MAX, ENS_T_FO = 0.6, 0.02, 15.0, 0.15


def batch_run(n: int, precision: str, floor: float, dev: int) -> dict:
    """One batched run of the ensemble: init, autotune, run; events/s counts
    events that completed (froze out or reached tau_max), failed events are
    reported apart."""
    import tempfile

    import numpy as np
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    from viral_b200.batch import Batch
    sides, bimp = ensemble_events(n)
    max_steps = C.steps_between(ENS_TAU0, ENS_TAU_MAX, ENS_DTAU)
    prec = A.PREC_MIXED if precision == "mixed" else A.PREC_FP64
    cfg = C.glauber_config(nx=8, ny=8, boost_invariant=True, precision=prec)
    t_init = time.perf_counter()
    B = Batch(cfg, sides, tau0=ENS_TAU0, dtau=ENS_DTAU, tau_max=ENS_TAU_MAX, t_freeze_gev=ENS_T_FO)
    npart = B.init_glauber(seeds=np.arange(n), bimp=bimp, efloor_gev=floor)
    t_init = time.perf_counter() - t_init
    _, ecc2_initial = B.observables()
    cache = os.path.join(tempfile.gettempdir(), "vh_batch_tuning.txt")
    t_tune = time.perf_counter()
    tune_ms = B.autotune(cache, probe_steps=16)
    t_tune = time.perf_counter() - t_tune
    tuning = B.tuning()
    with ClockSampler(dev) as clk:
        sec, graph = B.run(max_steps)
    tau, nst, st = B.events()
    eps_p_final, _ = B.observables()
    B.close()
    okev = st != 3
    done = int(np.sum((st == 1) | (st == 2)))
    cells = sides.astype(np.int64) ** 2
    return {"events_per_s": done / sec, "completed": done, "failed": int(np.sum(st == 3)),
            "running": int(np.sum(st == 0)), "frozen_out": int(np.sum(st == 1)), "tau_max": int(np.sum(st == 2)),
            "seconds": sec, "total_steps": int(np.sum(nst)), "cell_updates": float(np.sum(cells * nst)),
            "cell_updates_per_s": float(np.sum(cells * nst)) / sec,
            "steps_per_event": {"mean": float(np.mean(nst)), "min": int(nst.min()), "max": int(nst.max())},
            "graph": graph, "tuning": tuning, "autotune_ms_per_step": tune_ms, "autotune_seconds": t_tune,
            "init_seconds": t_init, "npart_mean": float(np.mean(npart)), "clocks": clk.summary(),
            "observables": {"eps2_initial_mean": float(np.mean(ecc2_initial)),
                            "eps_p_final_mean": float(np.mean(eps_p_final[okev])),
                            "corr_eps2_eps_p": float(np.corrcoef(ecc2_initial[okev], eps_p_final[okev])[0, 1])},
            "failed_events": [int(e) for e in np.where(st == 3)[0][:64]]}


def loop_fp64(n: int, per_side: int, floor: float) -> dict:
    """the single-event FP64 step looped over the ensemble's events one at a
    time, the maximum temperature read after every step as the reference's
    main loop does (NEWEST5/main.cpp:188-205); wall seconds per event on a
    stratified sample of `per_side` events per grid side, extrapolated by the
    side counts"""
    import numpy as np
    import torch
    from viral_b200 import configs as C
    sides, bimp = ensemble_events(n)
    max_steps = C.steps_between(ENS_TAU0, ENS_TAU_MAX, ENS_DTAU)
    per = {}
    for side in (64, 96, 128, 160, 200):
        ts = []
        for q in range(per_side):
            idx = np.where(sides == side)[0]
            ev = int(idx[q]) if len(idx) > q else q
            c = C.glauber_config(nx=side, ny=side, boost_invariant=True)
            inp = C.glauber_inputs(c, b=float(bimp[ev]), seed=ev, efloor_gev=floor)
            H = C.make_hydro(c, inp)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(max_steps):
                H.step(1)
                if H.max_temperature() < ENS_T_FO or H.tau >= ENS_TAU_MAX - 1e-9:
                    break
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            H.close()
        per[side] = float(np.mean(ts))
    seconds = float(sum(per[int(s_)] for s_ in sides))
    return {"events_per_s": n / seconds, "seconds_per_event_by_side": {str(k): v for k, v in per.items()},
            "extrapolated_seconds": seconds,
            "sample": f"{per_side} events per side, wall time, extrapolated by the side counts"}


def ensemble_record(args) -> dict:
    """c3: the batched ensemble of boost-invariant MC-Glauber events (grid side
    from {64,96,128,160,200}, dx = 0.1 fm, b uniform in [0,12] fm, seeds
    0..N-1, dtau = 0.02 fm/c from tau0 = 0.6 fm/c), each stopping when its
    maximum temperature falls below 0.15 GeV or at tau = 15 fm/c; one
    persistent kernel under a CUDA graph with the tuned variant, in mixed
    precision and in FP64, next to the single-event FP64 step looped over the
    events and the reference's CPU step on the host cores."""
    from viral_b200 import configs as C
    dev = int(os.environ.get("LOCAL_RANK", 0))
    n = args.ensemble_events
    floor = C.ENSEMBLE_FLOOR_GEV if args.ensemble_floor is None else args.ensemble_floor
    mixed = batch_run(n, "mixed", floor, dev)
    fp64 = batch_run(n, "fp64", floor, dev) if args.ensemble_fp64 else None
    loop = loop_fp64(n, args.loop_per_side, floor) if args.loop_per_side > 0 else None
    out = {"metric": "events/s", "value": mixed["events_per_s"], "unit": "events/s", "n_events": n,
           "what": "completed events (frozen out or tau_max) per device second of the batched run; failed events "
                   "(root-find or causality in the near-vacuum edge) counted apart",
           "batch_mixed": mixed, "batch_fp64": fp64, "loop_fp64": loop,
           "speedup_mixed_batch_vs_fp64_batch": (mixed["events_per_s"] / fp64["events_per_s"]) if fp64 else None,
           "speedup_mixed_batch_vs_fp64_loop": (mixed["events_per_s"] / loop["events_per_s"]) if loop else None,
           "config": {"workload": "glauber ensemble", "sides": [64, 96, 128, 160, 200], "dx_fm": 0.1,
                      "b_fm": [0, 12], "seeds": [0, n - 1], "dtau_fm": ENS_DTAU, "tau0_fm": ENS_TAU0,
                      "tau_max_fm": ENS_TAU_MAX, "t_freeze_gev": ENS_T_FO, "floor_gev_fm3": floor,
                      "eos": "synthetic table (2000 rows)", "eta_over_s": 0.08}}
    if args.cpu_seconds > 0:
        rates, procs, desc = reference_windows("ensemble", args.cpu_seconds, 1, reference_procs())
        cpu_seconds_total = mixed["cell_updates"] / rates[0]
        out["cpu_baseline"] = {"value": mixed["completed"] / cpu_seconds_total, "unit": "events/s", "cores": procs,
                               "kind": "reference", "cell_updates_per_s": rates[0],
                               "sample": f"{desc}, {args.cpu_seconds:.0f} s; the ensemble's "
                                         f"{mixed['cell_updates']:.4g} cell updates at that rate; {cpu_model()}"}
    return out


def ensemble(args):
    """standalone: the ensemble record alone (--ensemble N)"""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    args.ensemble_events = args.ensemble
    print(json.dumps(ensemble_record(args)), flush=True)


def ensemble_cpu_baseline(seconds: float, cell_steps: float, n_events: int) -> dict | None:
    """events/s of the reference's CPU step on the host cores for an ensemble
    of n_events that takes cell_steps interior cell updates in all: the
    reference's boost-invariant step on windows of an ensemble event, its
    aggregate cell-updates/s taken as the rate of the ensemble's events (the
    step's cost per cell does not depend on the grid side)"""
    if seconds <= 0:
        return None
    rates, cores, desc = reference_windows("ensemble", seconds, 1, reference_procs())
    return {"value": n_events * rates[0] / cell_steps, "unit": "events/s", "cores": cores, "kind": "reference",
            "cell_updates_per_s": rates[0], "sample": f"{desc}, {seconds:.0f} s; {cpu_model()}"}


# ---------------------------------------------------------------- adjoint


def adjoint_record(args) -> dict:
    """c4: discrete adjoint of the momentum anisotropy eps_p at tau = 7.2 fm/c
    of the boost-invariant 128x128 MC-Glauber event (dx = 0.1 fm, b = 7 fm,
    seed 0, floor 0.5 GeV/fm^3; 330 steps of 0.02 fm/c from 0.6 fm/c; eta/s =
    0.08 + 1.0 GeV^-1 max(T - 0.154 GeV, 0)), checkpoints every 25 steps, in
    FP64 and mixed precision.  The forward is vh_step(330) + vh_eps_p; the
    adjoint is one vh_adjoint_eps_p call (forward with checkpoints, segment
    recomputation, reverse steps, gradient export).  Device time from CUDA
    events on the handle's stream, the fastest of the repetitions (forward
    and adjoint alike: a shared box can slow a single repetition).  Both
    gradients are checked against central differences of the FP64 forward
    (h = 1e-6) along seeded unit directions in e0 and relative perturbations
    of (c0, c1)."""
    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    nsteps = args.adjoint_steps if args.adjoint_steps > 0 else C.ADJOINT_STEPS
    reps = max(3, args.adjoint_reps)
    res, grads = {}, {}
    inp = None
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
            for rep in range(2 + reps):  # two untimed warm-up repetitions
                reinit()
                tf, eps_f = timed(lambda: (H.step(nsteps), H.eps_p())[1])
                reinit()
                ta, out = timed(lambda: H.adjoint_eps_p(nsteps, args.checkpoint_every, want_state=False))
                if rep >= 2:
                    fwd.append(tf)
                    adj.append(ta)
            phases = H.adjoint_phase_times()
            res[name] = {"forward_ms": min(fwd), "adjoint_ms": min(adj), "ratio": min(adj) / min(fwd),
                         "repetitions": reps, "timing": "fastest of the repetitions, forward and adjoint alike",
                         "eps_p": out[0], "eps_p_forward": eps_f,
                         "adjoint_phases_ms": {"forward_with_checkpoints": phases[0], "recompute_with_records": phases[1],
                                               "reverse": phases[2], "rest": phases[3]},
                         "grad_etas": out[3].tolist(), "grad_e0_norm": float(np.linalg.norm(out[2]))}
            grads[name] = (out[2], out[3])
            H.close()
        if args.adjoint_fd > 0 and inp is not None:
            def eps_of(e0, c):
                cfg2 = C.adjoint_config(128, A.PREC_FP64, c[0], c[1])
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
            fd_dirs, dirs = [], []
            for _ in range(args.adjoint_fd):
                v = rng.normal(size=128 * 128)
                d = np.zeros_like(inp["e"])
                d[m] = v / np.linalg.norm(v)
                dirs.append(d)
                fd_dirs.append((eps_of(inp["e"] + h * d, c) - eps_of(inp["e"] - h * d, c)) / (2 * h))
            fd_c = []
            for k in range(2):
                cp = c.copy(); cm = c.copy()
                cp[k] *= 1 + h; cm[k] *= 1 - h
                fd_c.append((eps_of(inp["e"], cp) - eps_of(inp["e"], cm)) / (2 * h * c[k]))
            for name, (ge, gc) in grads.items():
                res[name]["fd_check"] = {
                    "h": h, "against": "central differences of the FP64 forward",
                    "e0_unit_directions_rel_err": [abs(float(np.dot(ge, d)) - f) / abs(f) for d, f in zip(dirs, fd_dirs)],
                    "c0_c1_rel_err": [abs(gc[k] - fd_c[k]) / abs(fd_c[k]) for k in range(2)]}
    first = "fp64" if "fp64" in res else "mixed"
    res["milne_3d"] = adjoint3_record(args, stream)
    return {"metric": "adjoint/forward time ratio", "value": res[first]["ratio"], "unit": "x",
            "higher_is_better": False, "dtype": "f64" if first == "fp64" else "f32 (FP64 implicit-function solve)",
            "mixed_ratio": res["mixed"]["ratio"] if "mixed" in res else None, "detail": res, "clocks": clk.summary(),
            "config": {"workload": "glauber_128x128 adjoint", "grid": [128, 128, 1], "b_fm": 7.0, "seed": 0,
                       "floor_gev_fm3": C.ADJOINT_FLOOR_GEV, "steps": nsteps, "tau_fm": [0.6, 0.6 + 0.02 * nsteps],
                       "eta_over_s": "0.08 + 1.0 max(T - 0.154, 0)", "checkpoint_every": args.checkpoint_every,
                       "observable": "eps_p"}}


def adjoint3_record(args, stream) -> dict:
    """The 3+1D adjoint on the benchmarked event's grid: 161x161x41 Milne
    cells (dx = 0.1 fm, d eta = 0.25), MC-Glauber b = 7 fm, seed 0, floor 0.5
    GeV/fm^3, eta/s = 0.08 + 1.0 GeV^-1 max(T - 0.154 GeV, 0); 20 steps from
    0.6 fm/c, checkpoints every 10; FP64 and mixed.  The gradient along two
    seeded unit directions of e0 and along (c0, c1) against central
    differences of the FP64 forward (h = 1e-4 for e0: the directional
    derivatives are small and rounding dominates at 1e-6; 1e-6 for c)."""
    import numpy as np
    import torch
    from viral_b200 import _abi as A
    from viral_b200 import configs as C
    nsteps, every, reps = 20, 10, 3
    out, grads = {}, {}
    inp = None

    def cfg_of(prec, c=(0.08, 1.0)):
        return C.glauber_config(nx=161, ny=161, nz=41, boost_invariant=False, precision=prec, etas0=c[0], etas1=c[1])

    for name, prec in (("fp64", A.PREC_FP64), ("mixed", A.PREC_MIXED)):
        cfg = cfg_of(prec)
        if inp is None:
            inp = C.glauber_inputs(cfg, b=7.0, seed=0, efloor_gev=C.ADJOINT_FLOOR_GEV)
        H = C.make_hydro(cfg, inp)
        A.check(A.lib().vh_set_stream(H.h, ctypes_void_p(stream.cuda_stream)), H.h)

        def reinit():
            H.init_profile(inp["tau"], inp["e"], inp["ux"], inp["uy"], inp["ueta"], inp["prevu"], inp["pi_mode"])
            torch.cuda.synchronize()

        def timed(fn):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), r

        fwd, adj = [], []
        for rep in range(2 + reps):
            reinit()
            tf, _ = timed(lambda: (H.step(nsteps), H.eps_p())[1])
            reinit()
            ta, r = timed(lambda: H.adjoint_eps_p(nsteps, every, want_state=False))
            if rep >= 2:
                fwd.append(tf)
                adj.append(ta)
        ph = H.adjoint_phase_times()
        H.close()
        out[name] = {"forward_ms": min(fwd), "adjoint_ms": min(adj), "ratio": min(adj) / min(fwd), "eps_p": r[0],
                     "adjoint_phases_ms": {"forward_with_checkpoints": ph[0], "recompute_with_records": ph[1],
                                           "reverse": ph[2], "rest": ph[3]}}
        grads[name] = (r[2], r[3])
    if args.adjoint_fd > 0:
        def eps_of(e0, c):
            with C.make_hydro(cfg_of(A.PREC_FP64, c), dict(inp, e=e0)) as H2:
                H2.step(nsteps)
                return H2.eps_p()
        gx, gy, gz = 167, 167, 47
        m = np.zeros((gz, gy, gx), bool)
        m[3:44, 3:164, 3:164] = True
        m = m.reshape(-1)
        rng = np.random.default_rng(4321)
        c = np.array([0.08, 1.0])
        dirs, fd = [], []
        for _ in range(2):
            v = rng.normal(size=int(m.sum()))
            d = np.zeros_like(inp["e"])
            d[m] = v / np.linalg.norm(v)
            dirs.append(d)
            fd.append((eps_of(inp["e"] + 1e-4 * d, c) - eps_of(inp["e"] - 1e-4 * d, c)) / 2e-4)
        fdc = []
        for k in range(2):
            cp = c.copy(); cm = c.copy()
            cp[k] *= 1 + 1e-6; cm[k] *= 1 - 1e-6
            fdc.append((eps_of(inp["e"], cp) - eps_of(inp["e"], cm)) / (2e-6 * c[k]))
        for name, (ge, gc) in grads.items():
            out[name]["fd_check"] = {
                "e0_unit_directions_rel_err": [abs(float(np.dot(ge, d)) - f) / abs(f) for d, f in zip(dirs, fd)],
                "c0_c1_rel_err": [abs(gc[k] - fdc[k]) / abs(fdc[k]) for k in range(2)]}
    out["config"] = {"workload": "glauber_161x161x41 adjoint (3+1D Milne)", "grid": [161, 161, 41], "b_fm": 7.0,
                     "seed": 0, "floor_gev_fm3": C.ADJOINT_FLOOR_GEV, "steps": nsteps, "checkpoint_every": every,
                     "eta_over_s": "0.08 + 1.0 max(T - 0.154, 0)", "observable": "eps_p over every eta slice"}
    return out


def adjoint_ratio(args):
    """standalone: the adjoint record alone (--adjoint)"""
    out = adjoint_record(args)
    out.update({"n_gpus": 1, "data": "synthetic (seeded MC-Glauber initial state)", "vs_baseline": None})
    print(json.dumps(out), flush=True)


def ctypes_void_p(v):
    import ctypes
    return ctypes.c_void_p(v)


# ---------------------------------------------------------------- arms


def reference_arm(args, world):
    """the reference's CPU step on the benchmarked workload (windows of its
    Glauber state, all host cores); rank 0 only"""
    t0 = time.perf_counter()
    procs = reference_procs()
    rates, procs, desc = reference_windows(args.workload, args.ref_sample_seconds, args.warmup + args.steps, procs)
    timed = rates[args.warmup:]
    value = statistics.mean(timed)
    sample = f"{desc}; each step a sample of about {args.ref_sample_seconds:.1f} s per process; {cpu_model()}"
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded MC-Glauber initial state)",
           "config": line_config(args.workload, "fp64", world),
           "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference", "sample": sample},
           "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "sample_rates": timed, "wall_s": time.perf_counter() - t0}
    print(json.dumps(out), flush=True)


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
        if rank == 0:
            reference_arm(args, world)
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    out = run_ours(args, rank, world, dist)
    if rank == 0 and world == 1 and "e2e" in out:
        subs = set(x for x in args.sub.split(",") if x and x != "none")
        if "mixed" in subs and args.precision == "fp64":
            out["mixed"] = mixed_record(args, out["ms_per_step"])
        if "ensemble" in subs:
            out["ensemble"] = ensemble_record(args)
        if "adjoint" in subs:
            out["adjoint"] = adjoint_record(args)
        if args.cpu_seconds > 0:
            rates, procs, desc = reference_windows(args.workload, args.cpu_seconds, 1, reference_procs())
            out["cpu_baseline"] = {"value": rates[0], "unit": METRIC, "cores": procs, "kind": "reference",
                                   "sample": f"{desc}; {args.cpu_seconds:.0f} s; {cpu_model()}"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
