"""Throughput of the coupled atmosphere-wildfire time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config hills8|hill|flat] [--precision fp32|fp64]

Metric: Mcell-steps/s = (Nx*Ny*Nz stored nodes) x steps / time.  A step is one
full RK4 time step (4 RHS stages, FP64 pressure Poisson solve, projection,
boundary rules, clamps) over the whole grid.  Default workload: the
mixed-precision configuration, 512 x 512 x 128 with 8 seeded hills, FP32
stencil + FP64 pressure (`hills8`); the plain FP64 path on the same grid is
timed beside it.  Data are seeded synthetic fields (no dataset exists for this
model).  The state (670 MB FP32, 1.3 GB FP64) is larger than the 126 MB L2,
so no explicit L2 flush is needed between timed steps.

Under torchrun (N > 1) every rank advances its own replica of the workload
(the single-domain step has no exchange to shard; replicas only) and the reported value
is the aggregate over ranks, timed as the max over ranks.

--impl reference times the reference's own CPU implementation (its src/cu
sources compiled for the host by oracle/Makefile, OpenMP over its virtual
threads) on the same full workload: W + K steps, the last K timed.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="hills8", choices=["hills8", "hill", "flat"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-refgpu", action="store_true", help="skip timing the reference's own GPU build")
    ap.add_argument("--ensemble", type=int, default=0, metavar="M",
                    help="instead: M seeded members of uneven grids (Nx, Ny in 96..256, Nz = 64), "
                         "one graph launch per ensemble step against the members stepped one by one")
    return ap.parse_args()


def build_params_only(name, **kw):
    """The parsed parameter record of a workload (terrain applied), without fields."""
    from wildfires_b200 import configs, read_parameters
    case = configs.CASES[name](**kw)
    d = tempfile.mkdtemp(prefix="wf_bench_")
    path = os.path.join(d, "parameters.txt")
    with open(path, "w") as f:
        f.write(configs.param_text(case.params))
    P = read_parameters(path)
    topo = case.topography(P)
    if topo is not None:
        P.set_topography(topo)
    return P


def build_case(name, **kw):
    from wildfires_b200 import configs, read_parameters
    case = configs.CASES[name](**kw)
    d = tempfile.mkdtemp(prefix="wf_bench_")
    path = os.path.join(d, "parameters.txt")
    with open(path, "w") as f:
        f.write(configs.param_text(case.params))
    P = read_parameters(path)
    topo = case.topography(P)
    if topo is not None:
        P.set_topography(topo)
    y0, p0 = case.fields(P)
    return case, P, y0, p0


def workload_config(name, P, prec, world):
    """The `config` object both arms print for the same workload."""
    r = P.rec
    S = 4 * r.Nx * r.Ny * r.Nz + r.Nx * r.Ny * r.Nz_Y_max
    return {"workload": workload_name(name, P, prec), "grid": [r.Nx, r.Ny, r.Nz], "cells": r.Nx * r.Ny * r.Nz,
            "dt": r.dt, "l2": "inputs larger than L2 (state %.0f MB), no flush" % (S * (4 if prec == "fp32" else 8) / 1e6),
            "parallelism": "replicas x%d" % world}


def workload_name(name, P, prec):
    r = P.rec
    form = "FP32 stencil + FP64 Poisson" if prec == "fp32" else "plain FP64"
    desc = {"hills8": "8 seeded gaussian hills", "hill": "single gaussian hill", "flat": "flat terrain"}[name]
    return "%s %dx%dx%d, %s, %s, RK4 dt=%g s" % (name, r.Nx, r.Ny, r.Nz, desc, form, r.dt)


# ---- clocks sampled during the timed region ----------------------------------
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 50 ms, started before
    the warm-up so that it is running when the timed region begins; stop()
    keeps the samples whose timestamps fall inside the timed window."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, window=None):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 10:
                    try:
                        ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    except ValueError:
                        ts = None
                    rows.append((ts, parts[1:]))
        os.unlink(self.out.name)
        if not rows:
            return None
        inside = [r for ts, r in rows if window and ts is not None and window[0] - 0.05 <= ts <= window[1] + 0.05]
        in_window = bool(inside)
        rows = inside if inside else [r for _, r in rows]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "samples_from": "timed window" if in_window else "whole run (no sample inside the timed window)"}


# ---- algorithmic bytes (roofline model) -------------------------------------
def kernel_bytes(name, P, prec):
    """Compulsory DRAM bytes per launch of each kernel kind.

    A state pass touches S = 4 N + N_Y values of s bytes.  Over the four RK4
    stages the fused stage kernel reads the stage input 3 times (stage 1 reads
    y_n, which is its input), y_n 4 times and the accumulator 3 times, and
    writes the accumulator 3 times and the stage output 4 times: 17 S values
    per step, 17/4 S per launch.  The pressure kernels move the half spectrum
    G = Nz (Nx-1) ((Ny-1)/2+1) complex FP64 values once in and once out.
    """
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    NY = r.Nx * r.Ny * r.Nz_Y_max
    s = 4 if prec == "fp32" else 8
    S = 4 * N + NY
    h1 = (r.Ny - 1) // 2 + 1
    G = (r.Nz) * (r.Nx - 1) * h1 * 16          # spectral slab incl. the top-plane slice
    return {
        "stage_fused": 17 * s * S / 4,
        "stage_utau": 0,
        "stage_bc": 0,
        # read u, v, w (+ top plane of p); write half spectrum
        "p_rhs_ffty": 3 * s * N + G,
        "p_fftx_fwd": 2 * G,
        "p_tridiag": 2 * G,
        "p_fftx_inv": 2 * G,
        # read half spectrum, write p
        "p_iffty_out": G + 8 * N,
        # read p, u, v, w, T, Y; write u, v, w
        "project": 8 * N + s * S + 3 * s * N,
    }.get(name, 0)


def step_model_bytes(P, prec):
    """Algorithmic bytes per cell-step of the whole step: 17 state passes of the
    RK4 stages, the pressure solve's spectral traffic and the projection."""
    r = P.rec
    s = 4 if prec == "fp32" else 8
    fY = r.Nz_Y_max / r.Nz
    return 17 * s * (4 + fY) + 3 * s + 152 + (8 + 6 * s)


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---- CPU reference ------------------------------------------------------------
def cpu_reference_sample(case_name, warmup=1, steps=1):
    """The reference's own solver on the host cores, on the full workload for a
    bounded number of steps (one warm-up step, one timed by the reference's
    own step timer: about 35 s of CPU work at 512 x 512 x 128 on 16 cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    from wildfires_b200 import configs
    if not ref_runner.available("host"):
        return None
    seconds, P = ref_runner.time_steps(configs.CASES[case_name](Nt=warmup + steps), warmup)
    r = P.rec
    cells = r.Nx * r.Ny * r.Nz
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"value": cells * steps / seconds / 1e6, "unit": METRIC, "cores": cores, "kind": "reference",
            "sample": "full %s workload %dx%dx%d, %d step timed after %d warm-up step (%.1f s), the reference's "
                      "own per-step timer" % (case_name, r.Nx, r.Ny, r.Nz, steps, warmup, seconds),
            "seconds": seconds, "steps": steps}


def reference_gpu_sample(case_name, n_short=2, n_long=10, repeats=2):
    """The reference's own sm_100a build (oracle/_ref/ref_gpu: its src/cu
    sources compiled unmodified, FP64) on the same workload and GPU: wall time
    of its solve_PDE for n_long and n_short steps; the difference divided by
    the extra steps removes its set-up (allocations, coefficient tables) and
    the state it writes at its last step.  Dirty pages are flushed before each
    run and the faster of `repeats` runs is kept, so that the write-back of
    one run's files does not land in another run's time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    from wildfires_b200 import configs
    if not ref_runner.available("gpu"):
        return None
    secs = {}
    for n in (n_short, n_long):
        best = None
        for _ in range(repeats):
            os.sync()
            t = ref_runner.run(configs.CASES[case_name](Nt=n), "time", flavour="gpu")["seconds"]
            best = t if best is None else min(best, t)
        secs[n] = best
    per = (secs[n_long] - secs[n_short]) / (n_long - n_short)
    P = build_params_only(case_name)
    cells = P.rec.Nx * P.rec.Ny * P.rec.Nz
    return {"value": round(cells / per / 1e6, 2), "unit": METRIC, "ms_per_step": round(per * 1e3, 2),
            "dtype": "f64", "how": "reference src/cu built for sm_100a, solve_PDE wall time for %d and %d steps "
                                   "(fastest of %d runs each), difference per step (set-up removed)"
                                   % (n_short, n_long, repeats)}


# ---- GPU arm --------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    from wildfires_b200 import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    case, P, y0, p0 = build_case(args.config)
    r = P.rec
    cells = r.Nx * r.Ny * r.Nz
    K, W = args.steps, args.warmup

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_steps(solver, K, clocks=None):
        stream = torch.cuda.ExternalStream(solver.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        solver.synchronize()
        t0 = time.time()
        e0.record(stream)
        solver.step(K)
        e1.record(stream)
        solver.synchronize()
        torch.cuda.synchronize()
        t1 = time.time()
        barrier()
        info = clocks.stop((t0, t1)) if clocks else None
        return e0.elapsed_time(e1), info

    res = {}
    sol = Solver(P, args.precision)
    sol.upload(y0, p0)
    clocks = ClockSampler(dev)
    clocks.start()
    sol.step(W)
    sol.synchronize()
    ms, clk = timed_steps(sol, K, clocks)
    ms = max_over_ranks(ms)
    ms_step = ms / K
    value = cells * K * world / (ms * 1e-3) / 1e6
    launches = sol.launches_per_step() * K * world   # all ranks' kernels in the timed region

    # per-kernel device times (eager launches with events on the solver stream)
    prof = sol.profile(2)
    total = sum(t for t, n in prof.values())
    dom = max(prof, key=lambda k: prof[k][0])
    t_dom, n_dom = prof[dom]
    avg_ms = t_dom / max(n_dom, 1)
    peak, peak_kind = peak_hbm()
    bytes_dom = kernel_bytes(dom, P, args.precision)
    achieved = bytes_dom / (avg_ms * 1e-3) / 1e9
    traf = traffic_table().get("%s/%s/%s" % (args.config, args.precision, dom))
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traf, "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": bytes_dom, "avg_launch_ms": round(avg_ms, 4),
                "share_of_step": round(t_dom / total, 4)}
    model = step_model_bytes(P, args.precision)
    step_roof = {"bytes_per_cell_step": round(model, 1),
                 "achieved_GBps": round(model * cells / (ms_step * 1e-3) / 1e9, 1)}
    step_roof["frac"] = round(step_roof["achieved_GBps"] / peak, 4)
    kernels = {k: {"ms_per_launch": round(t / max(n, 1), 4), "launches": n, "share": round(t / total, 4)}
               for k, (t, n) in prof.items()}
    y_fp32, _ = sol.download()
    steps_done = sol.time()[0]

    # end to end through the C-ABI with host buffers: H2D state, one step, D2H state
    pin_y = torch.empty(sol.S, dtype=torch.float64, pin_memory=True).numpy()
    pin_p = torch.empty(sol.N, dtype=torch.float64, pin_memory=True).numpy()
    pin_y[:] = y0
    pin_p[:] = p0
    from wildfires_b200 import _abi
    import ctypes as C
    L = _abi.lib()
    dp = C.POINTER(C.c_double)
    py, pp = pin_y.ctypes.data_as(dp), pin_p.ctypes.data_as(dp)
    ke = max(3, min(K, 10))

    def e2e_loop(upload, nsteps):
        for _ in range(nsteps):
            _abi.check(upload(sol._h, py, pp), "upload")
            _abi.check(L.wf_step(sol._h, 1), "step")
            _abi.check(L.wf_download_state(sol._h, py, pp), "download")

    # the state returned by each step is the next step's input (pinned host
    # buffers); wf_upload_state_async lets p's copy overlap the RK stages
    timings = {}
    for name, upload in (("blocking", L.wf_upload_state), ("async", L.wf_upload_state_async)):
        e2e_loop(upload, 2)
        pin_y[:] = y0
        pin_p[:] = p0
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_loop(upload, ke)
        torch.cuda.synchronize()
        timings[name] = max_over_ranks(time.perf_counter() - t0)
    h2d = sol.S * 8 + sol.N * 8
    e2e = {"value": round(cells * ke * world / timings["async"] / 1e6, 2), "unit": METRIC,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
           "blocking_upload_value": round(cells * ke * world / timings["blocking"] / 1e6, 2),
           "note": "per step: upload of the FP64 packed state and p from pinned host memory "
                   "(wf_upload_state_async: p's copy overlaps the RK stages), one step, download of "
                   "state and p; blocking_upload_value: the same with wf_upload_state"}
    stage_tile = sol.stage_tile()
    sol.close()

    # plain FP64 path on the same workload
    fp64 = None
    if not args.no_fp64 and args.precision == "fp32":
        s64 = Solver(P, "fp64")
        s64.upload(y0, p0)
        s64.step(W)
        s64.synchronize()
        ms64, _ = timed_steps(s64, K)
        ms64 = max_over_ranks(ms64)
        # bring the FP64 run to the same time level as the FP32 state
        n64 = s64.time()[0]
        if n64 < steps_done:
            s64.step(steps_done - n64)
        y64, _ = s64.download()
        s64.close()
        N = cells
        err = {}
        for q, nm in enumerate("uvwT"):
            a, b = y_fp32[q * N:(q + 1) * N], y64[q * N:(q + 1) * N]
            err[nm] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        nzy = P.nz_y()
        kk = np.arange(r.Nz_Y_max)[None, None, :]
        m = (kk < nzy[:, :, None]).reshape(-1)
        a, b = y_fp32[4 * N:][m], y64[4 * N:][m]
        err["Y"] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
        v64 = cells * K * world / (ms64 * 1e-3) / 1e6
        fp64 = {"value": round(v64, 2), "ms_per_step": round(ms64 / K, 4),
                "speedup_fp32_over_fp64": round(value / v64, 3),
                "fp32_rel_l2_vs_fp64_after_%d_steps" % steps_done: err}

    out = None
    if rank == 0:
        # the CPU baseline is a single-GPU figure: sampled on rank 0 of a 1-GPU run only
        cpu = None if (args.no_cpu or world > 1) else cpu_reference_sample(args.config)
        if cpu is None and not args.no_cpu and world == 1:
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                   "sample": "reference host build not available on this machine"}
        out = {
            "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded fields; no dataset exists for this model)",
            "config": workload_config(args.config, P, args.precision, world),
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "step_roofline": step_roof,
            "kernels": kernels, "cpu_baseline": cpu, "clocks": clk, "fp64": fp64,
            "stage_tile": "%dx%dx8 columns, %d threads per block (picked by the per-context tuner)" % stage_tile,
            "reference_gpu": None if (args.no_refgpu or world > 1) else reference_gpu_sample(args.config),
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


def run_reference(args):
    """The reference's own CPU implementation of the step (its src/cu sources
    built for the host by oracle/Makefile, OpenMP over its virtual threads, all
    host cores) on the FULL workload of the GPU arm: W + K steps in one run,
    the last K timed by the reference's own step timer.  The inputs are built
    with the reference's own parser and immersed-boundary precompute (the
    driver's params mode); this repository's library is not loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    from wildfires_b200 import configs
    if not ref_runner.available("host"):
        print(json.dumps({"impl": "reference", "unavailable": "reference host build (oracle/_ref/ref_host) not present"}))
        return None
    K, W = args.steps, args.warmup
    case = configs.CASES[args.config](Nt=W + K)
    seconds, P = ref_runner.time_steps(case, W)
    r = P.rec
    cells = r.Nx * r.Ny * r.Nz
    value = cells * K / seconds / 1e6
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    sample = ("full %s workload %dx%dx%d, %d timed steps after %d warm-up steps (%.1f s), the reference's own "
              "per-step timer" % (args.config, r.Nx, r.Ny, r.Nz, K, W, seconds))
    cfg = workload_config(args.config, P, args.precision, int(os.environ.get("WORLD_SIZE", "1")))
    cfg["workload"] = workload_name(args.config, P, "fp64")
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": METRIC,
           "n_gpus": args.gpus, "steps": K, "warmup": W, "ms_per_step": round(seconds / K * 1e3, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded fields)", "config": cfg,
           "cpu_baseline": {"value": round(value, 4), "unit": METRIC, "cores": cores, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": round(value, 4), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return out


def run_ensemble(args):
    """Ensemble throughput.  --ensemble M: M seeded members per GPU (weak
    scaling), partitioned across ranks by cells x steps with no collective
    while stepping.  On each rank: all of its members per step in one graph
    launch (concurrent member branches), then the same members stepped one
    after another (a graph launch and a wait each) for comparison."""
    import torch
    import torch.distributed as dist
    from wildfires_b200 import Ensemble, configs
    from wildfires_b200.sharding import partition
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    members = configs.ensemble(args.ensemble * world, Nt=300)
    costs = [m.params["Nx"] * m.params["Ny"] * m.params["Nz"] for m in members]
    mine = partition(costs, world)[rank]
    built = [configs.materialize(members[i]) for i in mine]
    cells_local = sum(P.rec.Nx * P.rec.Ny * P.rec.Nz for P, _, _ in built)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with Ensemble([b[0] for b in built], args.precision) as ens:
        for i, (P, y0, p0) in enumerate(built):
            ens[i].upload(y0, p0)
        ens.step(args.warmup)
        for m in ens.members:
            m.step(args.warmup)
        ens.synchronize()
        clk = ClockSampler(local) if rank == 0 else None
        if clk:
            clk.start()
            time.sleep(0.3)
        # ensemble steps: CUDA events on the stream the step graphs are launched on
        master = torch.cuda.ExternalStream(ens.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        w0 = time.time()
        t0 = time.perf_counter()
        e0.record(master)
        ens.step(args.steps)
        e1.record(master)
        ens.synchronize()
        wall_ens = time.perf_counter() - t0
        w1 = time.time()
        t_ens = max_over_ranks(e0.elapsed_time(e1) * 1e-3)
        barrier()
        # the same members one after another: each step event-timed on its own
        # stream (device time of the member's step graph) and, separately, the
        # wall clock of the whole serial loop (a launch and a wait per member step)
        gpu_ser = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for m in ens.members:
                st = torch.cuda.ExternalStream(m.stream())
                a0 = torch.cuda.Event(enable_timing=True)
                a1 = torch.cuda.Event(enable_timing=True)
                a0.record(st)
                m.step(1)
                a1.record(st)
                m.synchronize()
                gpu_ser += a0.elapsed_time(a1) * 1e-3
        wall_ser = max_over_ranks(time.perf_counter() - t0)
        t_ser = max_over_ranks(gpu_ser)
        clocks = clk.stop((w0, w1)) if clk else None
    cells = cells_local
    if world > 1:
        t = torch.tensor([float(cells_local)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        cells = int(t.item())
        dist.destroy_process_group()
    if rank != 0:
        return None
    v_ens = cells * args.steps / t_ens / 1e6
    v_ser = cells * args.steps / t_ser / 1e6
    out = {"metric": "ensemble Mcell-steps/s", "value": round(v_ens, 2), "unit": "Mcell-steps/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ens / args.steps * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32+f64" if args.precision == "fp32" else "f64", "data": "synthetic (seeded members)",
           "config": {"workload": "ensemble of %d members per GPU, Nx, Ny in {96..256}, Nz = 64, %s"
                                  % (args.ensemble, args.precision),
                      "members": len(members), "cells": cells,
                      "parallelism": "members partitioned over %d ranks, no collective while stepping" % world},
           "serial": {"value": round(v_ser, 2), "ms_per_step": round(t_ser / args.steps * 1e3, 3),
                      "wall_ms_per_step": round(wall_ser / args.steps * 1e3, 3),
                      "how": "each member: one graph launch per step, then a wait, members one after another; "
                             "ms_per_step sums the members' event-timed step graphs (device time, no gaps), "
                             "wall_ms_per_step is the host clock of the loop"},
           "speedup_over_serial": round(t_ser / t_ens, 3),
           "speedup_over_serial_wall": round(wall_ser / wall_ens, 3),
           "timing": "CUDA events on the launching streams, max over ranks", "clocks": clocks}
    print(json.dumps(out), flush=True)
    return out


def main():
    args = parse_args()
    if args.ensemble:
        run_ensemble(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
