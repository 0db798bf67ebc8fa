#!/usr/bin/env python
"""Benchmark of the AWFL Euler-3D ADER/WENO step on B200: Mcell-steps/s at 256x256x128.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp32|fp64] [--ord 5|9]

A "step" is one ADER time step (three directional splits, Temporal_ader::timeStep) of
the whole 256x256x128 grid. Workload: the rising thermal bubble scale-up case (cosine-
squared theta bubble +3 K, radius 2 km, centred at (10, 10, 2) km in a 20x20x10 km domain,
periodic x/y, walls in z, ord 5 / ngll 3, CFL 0.8) with seeded uniform +-0.01 K theta noise;
synthetic initial data generated on the device.

Our arm times K steps of the FP32 precision form (the headline `value`) and of the plain
FP64 path (`fp64`), each with CUDA events on the launching stream after W warm-up steps,
barrier + synchronize on both sides, max over ranks, and reports the FP32-vs-FP64 relative
L2 after 100 steps, the cost of the discrete adjoint against the forward step
(`adjoint`, FP64 at 128x128x64, 200 steps, checkpoint every 20), and the batching form
(`ensemble`: 64 FP32 members of uneven sizes, 50 steps, persistent kernels in a CUDA graph),
the 512x512x128 precision configuration (`precision`) and the same grid at ord 9 / ngll 5
(`ord9`: both forms' throughput and their relative L2 after 100 steps). The state (357 MB in FP64) is larger
than the 126 MB L2, so no flush is needed between steps. N > 1 runs N independent
replicas (one grid per GPU, no collective): the single-domain path has no exchange step.

Printed on rank 0: one JSON line; `tracers` adds the cost of the tracer transport (FP64,
three tracers) on the same grid.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s at 256²×128: FP32 vs plain FP64 (rel L2≤1e-5); adjoint/fwd"
UNIT = "Mcell-steps/s"
DATA = ("synthetic: cosine-squared theta bubble +3 K, radius 2 km, centre (10,10,2) km, "
        "+ seeded uniform +-0.01 K theta noise (splitmix64, seed 20261203)")
BUBBLE = dict(kind=1, shape=1, x0=10000.0, y0=10000.0, z0=2000.0, xrad=2000.0, yrad=2000.0,
              zrad=2000.0, amp=3.0, pwr=1.0, noise_amp=0.01, noise_seed=20261203)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--ord", type=int, default=5, choices=[5, 9])
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost leg")
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--adj-ckpt", type=int, default=20)
    ap.add_argument("--no-ensemble", action="store_true", help="skip the ensemble (batching) leg")
    ap.add_argument("--ens-members", type=int, default=64)
    ap.add_argument("--ens-steps", type=int, default=50)
    ap.add_argument("--no-precision", action="store_true", help="skip the 512x512x128 precision leg")
    ap.add_argument("--no-ord9", action="store_true", help="skip the ord-9 leg (256x256x128, ngll 5)")
    ap.add_argument("--no-tracers", action="store_true", help="skip the tracer-transport leg")
    ap.add_argument("--only", choices=["adjoint", "ensemble", "precision", "ord9", "tracers"],
                    help="run only that leg and print its JSON object (profiling aid)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the FP64 comparison arm and the 100-step accuracy check")
    return ap.parse_args()


def max_over_ranks(x, world):
    """The largest of every rank's value (the slowest replica's time): an all-reduce on the
    process group's device (CUDA tensor for NCCL, host tensor for gloo); x itself at N = 1."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def job_throughput(world, cells, steps, max_ms):
    """Whole-job Mcell-steps/s at N GPUs (weak scaling): every rank advances its `cells`
    cells `steps` times (its slab of the N-slab grid); the job takes the slowest rank's
    time."""
    return world * cells * steps / (max_ms * 1e-3) / 1e6


def cfl_for(ord_):
    # The driver's CFL 0.8 (driver.cpp:46). At ord 9 the reference's own scheme diverges
    # at 0.8 (NaN within 8 steps, reproduced with its code), so ord 9 runs at 0.4.
    return 0.8 if ord_ == 5 else 0.4


def bench_config(a):
    """The workload, identical in both arms (the arithmetic type is the line's dtype)."""
    h2 = a.ord - 1  # two halos of (ord-1)/2 cells
    mb = 5 * (a.nx + h2) * (a.ny + h2) * (a.nz + h2) * 8 / 1e6
    return {"workload": workload_name(a), "nx": a.nx, "ny": a.ny, "nz": a.nz, "ord": a.ord,
            "l2": "inputs larger than L2: the state is %.0f MB (FP64, or FP32 values + compensations) "
                  "> 126 MB, no flush" % mb}


def workload_name(a):
    return "rising thermal bubble %dx%dx%d, ord %d / ngll %d, CFL %.1f" % (
        a.nx, a.ny, a.nz, a.ord, 3 if a.ord == 5 else 5, cfl_for(a.ord))


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0) for r in rows)}


# ----------------------------------------------------------------------------- CPU baseline
def cpu_baseline(a, budget_s=20.0):
    """The reference's own CPU code (oracle/_ref, built from its sources on the project's
    stand-ins) with all host threads, on the same workload, a bounded number of steps."""
    from oracle import pyoracle
    cores = os.cpu_count() or 1
    kind = "reference" if pyoracle.ref_available(a.ord) else "port"
    if kind == "reference":
        R = pyoracle.RefHarness(a.nx, a.ny, a.nz, ord_=a.ord)
        R.init_state()
        R.set_bubble(1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
        R.add_theta_noise(20261203, 0.01)
        dt = R.compute_dt(cfl_for(a.ord))
        step = lambda: R.time_step(dt)  # noqa: E731
    else:
        O = pyoracle.Oracle(a.nx, a.ny, a.nz, ord_=a.ord)
        st = O.new_state()
        O.init_state(st)
        O.set_bubble(st, 1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
        O.add_theta_noise(st, 20261203, 0.01)
        dt = O.compute_dt(st, cfl_for(a.ord))
        step = lambda: O.time_step(st, dt)  # noqa: E731
    n, t0 = 0, time.perf_counter()
    while True:
        step()
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s or n >= 50 or (n >= 1 and el * (n + 1) / n > 2.5 * budget_s):
            break
    cells = a.nx * a.ny * a.nz
    return {"value": round(cells * n / el / 1e6, 4), "unit": UNIT, "cores": cores, "kind": kind,
            "sample": "%d full time steps of the %dx%dx%d workload, FP64, OpenMP %d threads, %.1f s"
                      % (n, a.nx, a.ny, a.nz, cores, el)}


# ----------------------------------------------------------------------------- reference arm
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import pyoracle
    cores = os.cpu_count() or 1
    if not pyoracle.ref_available(a.ord):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (the reference built from its sources) is not present; run build()"}))
        return 0
    cells = a.nx * a.ny * a.nz
    R = pyoracle.RefHarness(a.nx, a.ny, a.nz, ord_=a.ord)
    R.init_state()
    R.set_bubble(1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
    R.add_theta_noise(20261203, 0.01)
    dt = R.compute_dt(cfl_for(a.ord))
    # each step is one full time step of the workload (about 1 s on 16 host threads at
    # 256x256x128), so the default --steps 20 --warmup 3 ends in well under a minute
    t0 = time.perf_counter()
    R.time_step(dt)
    one = time.perf_counter() - t0
    for _ in range(max(0, a.warmup - 1)):
        R.time_step(dt)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        R.time_step(dt)
    el = time.perf_counter() - t0
    value = cells * a.steps / el / 1e6
    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(el / a.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
            "config": bench_config(a),
            "impl": "reference", "impl_note": "the reference's own code (oracle/_ref) on the host cores "
                                              "with OpenMP, rank 0 only",
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": "%d full time steps after %d warm-up, first step %.2f s" % (a.steps, a.warmup, one)},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- our arm
def make_domain(a, prec, local, world):
    """N = 1: the workload's grid on this GPU. N > 1: slab `rank` of one grid N times as
    long in x (a.nx cells of it per GPU, x extent and dx scaled alike), decomposed over the
    ranks with the halo-column exchange before every x split (SlabDomain)."""
    from awflcloud_b200 import capi
    if world == 1:
        ctx = capi.Context(a.nx, a.ny, a.nz, ord_=a.ord, precision=prec, device=local)
        st = ctx.new_state()
        ctx.init_state(st, **BUBBLE)
        dt = ctx.cfl(st, cfl_for(a.ord))
        return ctx, st, dt, ctx.split, ctx.step, lambda: ctx.dimswitch, lambda v: setattr(ctx, "dimswitch", v)
    from awflcloud_b200.slab import SlabDomain
    dom = SlabDomain(a.nx * world, a.ny, a.nz, device=local, xlen=20000.0 * world, ord_=a.ord, precision=prec)
    st = dom.new_state()
    dom.ctx.init_state(st, **BUBBLE)
    dt = dom.cfl(st, cfl_for(a.ord))
    return (dom.ctx, st, dt, lambda s, dt_, d: dom.split(s, dt_, d), lambda s, dt_: dom.step(s, dt_),
            lambda: dom.dimswitch, lambda v: setattr(dom, "dimswitch", v))


def time_form(a, prec, local, world, clocks=None):
    """Time K fused steps of one precision form; per-launch CUDA events on the stream."""
    import torch
    import torch.distributed as dist
    from awflcloud_b200 import capi, flops
    cells = a.nx * a.ny * a.nz
    ctx, st, dt, split, step, get_ds, set_ds = make_domain(a, prec, local, world)
    stream = torch.cuda.current_stream()
    peak = capi.measure_fma_peak(prec, local)
    peaks = {"peak_scalar": round(peak, 3)}
    if prec == capi.FP32:
        # sm_100's paired FP32 FMA retires two lanes per instruction: the pipe's ceiling is
        # the larger of the two measured rates
        paired = capi.measure_fma_peak(capi.PEAK_FP32_PAIRED, local)
        peaks["peak_paired"] = round(paired, 3)
        peak = max(peak, paired)
    for _ in range(a.warmup):
        step(st, dt)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.start()
    # Events between the three split launches of every step give the per-launch time of
    # the sweep kernel (the only kernel in the step at N = 1; at N > 1 the x split's
    # interval also holds the column packing and exchange).
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * a.steps + 1)]
    ev[0].record(stream)
    for s in range(a.steps):
        ds = get_ds()
        for spl in range(3):
            split(st, dt, spl if ds else 2 - spl)
            ev[3 * s + spl + 1].record(stream)
        set_ds(1 - ds)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks is not None else None
    total_ms = ev[0].elapsed_time(ev[-1])
    launch_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(3 * a.steps)]
    max_ms = max_over_ranks(total_ms, world)
    fl = flops.flops_per_cell_step(a.ord)
    flops_launch = fl["flops"] / 3.0 * cells  # per split launch, averaged over directions
    avg_launch_s = statistics.mean(launch_ms) * 1e-3
    achieved = flops_launch / avg_launch_s / 1e12
    esz = 8 if prec == capi.FP64 else 4
    per_cell = EXECUTED_OPS.get((prec, a.ord), {}).get("ops_per_cell")
    ops_exec = per_cell * cells if per_cell else None
    roofline = {"bound": "fp64" if prec == capi.FP64 else "fp32",
                "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": TRAFFIC.get((prec, a.ord)),
                "peak_source": "measured in this run: awfl_measure_fma_peak (FMA chains, 2 flops per "
                               "FMA lane; FP32: the larger of scalar and paired FMA)",
                **peaks,
                "ops_algorithmic": flops_launch,
                "ops_executed": ops_exec,
                "frac_executed": round(ops_exec / avg_launch_s / 1e12 / peak, 4) if ops_exec else None,
                "ops_executed_source": EXECUTED_OPS.get((prec, a.ord), {}).get("source"),
                "launch_ms_avg": round(avg_launch_s * 1e3, 4),
                "bytes_algorithmic_per_launch": cells * 10 * esz * (1 if prec == capi.FP64 else 2)}
    return {"ctx": ctx, "state": st, "dt": dt, "step": step, "value": job_throughput(world, cells, a.steps, max_ms),
            "ms_per_step": max_ms / a.steps, "roofline": roofline, "clocks": clk, "flops": fl,
            "finite": bool(torch.isfinite(st).all().item())}


# DRAM bytes per sweep launch (read + write, mean over x/y/z): ncu's
# dram__bytes_read.sum + dram__bytes_write.sum of the sweep kernels on this 256x256x128
# workload (one capture of the same build; ncu cannot run inside the timed process).
TRAFFIC = {(0, 5): 650_500_000, (1, 5): 635_700_000}
# Floating-point operations the sweep kernels execute per cell and split (mean over x/y/z),
# from ncu's per-opcode thread-instruction counters on 256x256x64 (4,194,304 cells): FP32
# form: FADD + FMUL + 2 x FFMA, paired instructions counted per lane; FP64: DADD + DMUL +
# 2 x DFMA (the division and pow sequences included). The algorithmic count (flops.py)
# follows the reference's loops instead.
EXECUTED_OPS = {
    (1, 5): {"ops_per_cell": 1769, "source": "ncu sm__sass_thread_inst_executed_op_{fadd,fmul,ffma,fadd2,fmul2,"
                                             "ffma2}_pred_on, sweep kernels at 256x256x64"},
    (0, 5): {"ops_per_cell": 4766, "source": "ncu sm__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on, "
                                             "sweep kernels at 256x256x64"},
}


def rel_l2_after(a, steps, local):
    """FP32 form vs FP64 path after `steps` steps from the same initial data: relative L2
    per variable (interior cells)."""
    import torch
    from awflcloud_b200 import capi
    c64 = capi.Context(a.nx, a.ny, a.nz, ord_=a.ord, precision=capi.FP64, device=local)
    c32 = capi.Context(a.nx, a.ny, a.nz, ord_=a.ord, precision=capi.FP32, device=local)
    s64, s32 = c64.new_state(), c32.new_state()
    c64.init_state(s64, **BUBBLE)
    c32.init_state(s32, **BUBBLE)
    dt = c64.cfl(s64, cfl_for(a.ord))
    for _ in range(steps):
        c64.step(s64, dt)
        c32.step(s32, dt)
    h = c64.hs
    out = []
    for v in range(5):
        x = s32[v, h:-h, h:-h, h:-h].double()
        y = s64[v, h:-h, h:-h, h:-h]
        out.append((torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item())
    return out


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), GB/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (copy, read+write)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def output_leg(ctx, st, reps=20):
    """The output diagnostics kernel (Spatial::output's six fields, one launch) on the timed
    state: HBM-bound, so reported as algorithmic GB/s against the measured copy bandwidth.
    Algorithmic bytes per cell: the state read (5 FP64 values, or 5 FP32 values + 5 FP32
    compensations: 40 B) + 6 FP64 fields written (48 B)."""
    import torch
    cells = ctx.nx * ctx.ny * ctx.nz
    out = torch.empty((6, ctx.nz, ctx.ny, ctx.nx), dtype=torch.float64, device=st.device)
    for _ in range(3):
        ctx.output_fields(st, out)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        ctx.output_fields(st, out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nbytes = cells * (40 + 48)
    peak, src = hbm_peak()
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"kernel": "output_fields_kernel", "ms_per_launch": round(ms, 4), "bytes_algorithmic": nbytes,
            "achieved_gbs": round(gbs, 1), "peak_gbs": peak, "frac": round(gbs / peak, 4), "peak_source": src,
            "l2": "357 MB state + 403 MB fields > 126 MB L2"}


def ord9_leg(a, local):
    """The same grid and bubble at WENO ord 9 / ngll 5 (CFL 0.4): FP32 form and FP64 path
    throughput (K steps after W warm-up steps each) and their relative L2 after 100 steps."""
    import copy
    from awflcloud_b200 import capi
    b = copy.copy(a)
    b.ord = 9
    b.steps = min(a.steps, 10)
    r32 = time_form(b, capi.FP32, local, 1)
    r64 = time_form(b, capi.FP64, local, 1)
    errs = rel_l2_after(b, 100, local)
    pick = lambda r: {"value": round(r["value"], 3), "ms_per_step": round(r["ms_per_step"], 4),
                      "roofline_frac": r["roofline"]["frac"], "roofline_bound": r["roofline"]["bound"],
                      "finite": r["finite"]}
    return {"workload": "rising thermal bubble %dx%dx%d, ord 9 / ngll 5, CFL 0.4" % (b.nx, b.ny, b.nz),
            "steps": b.steps, "warmup": b.warmup, "fp32": pick(r32), "fp64": pick(r64),
            "fp32_over_fp64": round(r32["value"] / r64["value"], 3),
            "flops_per_cell_step": r32["flops"]["flops"],
            "rel_l2_fp32_vs_fp64_after_100_steps": dict(zip(["rho", "rho_u", "rho_v", "rho_w", "rho_theta"], errs))}


def tracers_leg(a, local, ntr=3, steps=5, warmup=2):
    """Tracer transport (the reference's compiled-out tracer code, built in) on the main grid
    with the driver's three positive-definite tracers, awfl_step_tracers vs awfl_step, CUDA
    events on the launching stream: the FP64 path, and the FP32 form (FP32 reconstruction,
    fluxes and limiter, FP64 tracer arrays)."""
    import torch
    from awflcloud_b200 import capi
    stream = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def dense(tr):
        # tracers 1 and 2 made nonzero everywhere: rho times smooth positive fields of x, z and y
        hs = (a.ord - 1) // 2
        dev = tr.device
        x = (torch.arange(a.nx + 2 * hs, device=dev, dtype=torch.float64) - hs + 0.5) / a.nx
        y = (torch.arange(a.ny + 2 * hs, device=dev, dtype=torch.float64) - hs + 0.5) / a.ny
        z = (torch.arange(a.nz + 2 * hs, device=dev, dtype=torch.float64) - hs + 0.5) / a.nz
        tr[1] = tr[0] * (1 + 0.5 * torch.sin(2 * math.pi * x)[None, None, :] * torch.sin(math.pi * z)[:, None, None])
        tr[2] = tr[0] * (1 + 0.5 * torch.cos(2 * math.pi * y)[None, :, None])

    def form(prec, fill=None):
        c = capi.Context(a.nx, a.ny, a.nz, ord_=a.ord, precision=prec, device=local)
        st = c.new_state()
        c.init_state(st, kind=capi.INIT_BUBBLE, noise_amp=0.01)
        tr = c.new_tracers(ntr)
        c.init_tracers(tr)
        if fill is not None:
            fill(tr)
        dt = c.cfl(st, cfl_for(a.ord))
        ms_tr = timed(lambda: c.step_tracers(st, tr, dt))
        ms_plain = timed(lambda: c.step(st, dt))
        finite = bool(torch.isfinite(tr).all().item())
        del c, st, tr
        return ms_tr, ms_plain, finite

    ms_tr, ms_plain, finite = form(capi.FP64)
    ms_tr32, ms_plain32, finite32 = form(capi.FP32)
    ms_trd, ms_plaind, finited = form(capi.FP64, dense)
    ms_trd32, ms_plaind32, finited32 = form(capi.FP32, dense)
    cells = a.nx * a.ny * a.nz
    return {"workload": "%s, FP64, %d positive-definite tracers (uniform, theta, block)" % (workload_name(a), ntr),
            "steps": steps, "warmup": warmup, "ms_per_step_with_tracers": round(ms_tr, 4),
            "ms_per_step_without": round(ms_plain, 4), "tracer_ms_per_step": round(ms_tr - ms_plain, 4),
            "value": round(cells / (ms_tr * 1e-3) / 1e6, 3), "unit": "Mcell-steps/s", "finite": finite,
            "fp32": {"ms_per_step_with_tracers": round(ms_tr32, 4), "ms_per_step_without": round(ms_plain32, 4),
                     "tracer_ms_per_step": round(ms_tr32 - ms_plain32, 4),
                     "value": round(cells / (ms_tr32 * 1e-3) / 1e6, 3), "finite": finite32},
            "dense": {"tracers": "uniform; rho*(1 + 0.5 sin(2 pi x/Lx) sin(pi z/Lz)); rho*(1 + 0.5 cos(2 pi y/Ly)): "
                                 "nonzero everywhere, so no stencil of zeros skips its reconstruction",
                      "fp64": {"ms_per_step_with_tracers": round(ms_trd, 4),
                               "tracer_ms_per_step": round(ms_trd - ms_plaind, 4), "finite": finited},
                      "fp32": {"ms_per_step_with_tracers": round(ms_trd32, 4),
                               "tracer_ms_per_step": round(ms_trd32 - ms_plaind32, 4), "finite": finited32}},
            "note": "per split: the state's fused sweep recording the density / normal-momentum ADER series, "
                    "the pre-split density, reciprocal densities and per face the Riemann mass flux, upwind velocity "
                    "and density; then the tracer launches (cell with the upwind fluxes, limiter faces, limiter "
                    "lines, update); tracers divided by the density once per step, kept divided between splits"}


def adjoint_leg(a, local):
    """Cost of the discrete adjoint against the forward step (FP64, ord 5, 128x128x64,
    same bubble): the forward pass of a gradient computation (adj_steps steps, a state
    checkpoint every adj_ckpt steps) and its backward pass (awfl_step_adjoint once per
    segment, last segment first, each recomputing its segment from the checkpoint), both
    timed with CUDA events on the stream."""
    import torch
    from awflcloud_b200 import capi
    n = (128, 128, 64)
    ctx = capi.Context(*n, ord_=5, precision=capi.FP64, device=local)
    s0 = ctx.new_state()
    ctx.init_state(s0, **BUBBLE)
    dt = ctx.cfl(s0, 0.8)
    nseg = (a.adj_steps + a.adj_ckpt - 1) // a.adj_ckpt
    ckpts = [torch.empty_like(s0) for _ in range(nseg)]
    lam = torch.empty_like(s0)
    stream = torch.cuda.current_stream()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def forward():
        s = s0.clone()
        ctx.dimswitch = 1
        ds = []
        for k in range(a.adj_steps):
            if k % a.adj_ckpt == 0:
                ckpts[k // a.adj_ckpt].copy_(s)
                ds.append(ctx.dimswitch)
            ctx.step(s, dt)
        return s, ds

    def backward(sN, ds):
        lam.copy_(sN)  # dJ/dS_end for J = 1/2 |S_end|^2
        for g in range(nseg - 1, -1, -1):
            ctx.dimswitch = ds[g]
            ctx.step_adjoint(ckpts[g], lam, min(a.adj_ckpt, a.adj_steps - g * a.adj_ckpt), dt)

    sN, ds = forward()  # warm-up (and tape allocation)
    backward(sN, ds)
    torch.cuda.synchronize()
    e[0].record(stream)
    sN, ds = forward()
    e[1].record(stream)
    backward(sN, ds)
    e[2].record(stream)
    torch.cuda.synchronize()
    fwd_ms, adj_ms = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    g1 = lam.clone()
    tape1 = ctx.adjoint_tape_bytes(a.adj_ckpt)
    # two-level: every segment taken one step at a time (a plain forward pass keeps the
    # state at every step, then each step is recorded and reversed, last first)
    ctx.set_adjoint_subwindow(1)
    backward(sN, ds)  # warm-up of the smaller tape
    torch.cuda.synchronize()
    e[1].record(stream)
    backward(sN, ds)
    e[3].record(stream)
    torch.cuda.synchronize()
    adj2_ms = e[1].elapsed_time(e[3])
    tape2 = ctx.adjoint_tape_bytes(a.adj_ckpt)
    same = bool(torch.equal(g1, lam))
    ctx.set_adjoint_subwindow(0)
    return {"workload": "rising bubble 128x128x64, ord 5, FP64, %d steps, checkpoint every %d"
                        % (a.adj_steps, a.adj_ckpt),
            "fwd_ms_per_step": round(fwd_ms / a.adj_steps, 4), "adj_ms_per_step": round(adj_ms / a.adj_steps, 4),
            "adj_over_fwd": round(adj_ms / fwd_ms, 3),
            "tape_bytes": tape1,
            "two_level": {"subwindow_steps": 1, "adj_ms_per_step": round(adj2_ms / a.adj_steps, 4),
                          "adj_over_fwd": round(adj2_ms / fwd_ms, 3), "tape_bytes": tape2,
                          "tape_reduction": round(tape1 / tape2, 2), "gradient_identical": same},
            "finite": bool(torch.isfinite(lam).all().item()),
            "note": "backward = recomputation of every segment from its checkpoint + reverse sweeps"}


def precision_leg(a, local):
    """The precision configuration: 512x512x128, ord 5, bubble amp 2 K radius 1.5 km +
    N(0, 0.05 K) theta noise (Box-Muller on splitmix64), 100 steps of the FP32 form and of
    the FP64 path from the same initial data: relative L2 per variable, and each form's
    change of the total perturbation mass (FP64 sums, awfl_state_sums)."""
    import numpy as np
    import torch
    from awflcloud_b200 import capi
    n, steps = (512, 512, 128), 100
    spec = dict(kind=1, shape=1, x0=10000.0, y0=10000.0, z0=2000.0, xrad=1500.0, yrad=1500.0, zrad=1500.0,
                amp=2.0, pwr=1.0, noise_amp=0.05, noise_seed=20261203, noise_kind=capi.NOISE_NORMAL)
    c64 = capi.Context(*n, precision=capi.FP64, device=local)
    c32 = capi.Context(*n, precision=capi.FP32, device=local)
    s64, s32 = c64.new_state(), c32.new_state()
    c64.init_state(s64, **spec)
    c32.init_state(s32, **spec)
    dt = c64.cfl(s64, 0.8)
    m64, m32 = c64.state_sums(s64)[0], c32.state_sums(s32)[0]
    for _ in range(steps):
        c64.step(s64, dt)
        c32.step(s32, dt)
    h = c64.hs
    errs = {}
    for v, name in enumerate(("rho", "rho_u", "rho_v", "rho_w", "rho_theta")):
        x = s32[v, h:-h, h:-h, h:-h].double()
        y = s64[v, h:-h, h:-h, h:-h]
        errs[name] = (torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)).item()
    dv = (20000.0 / n[0]) * (20000.0 / n[1]) * (10000.0 / n[2])
    total = float(np.sum(c64.background()["hyDensCells"][h:-h])) * n[0] * n[1] * dv
    return {"workload": "512x512x128, ord 5, bubble 2 K / 1.5 km + N(0, 0.05 K) theta noise, %d steps" % steps,
            "rel_l2_fp32_vs_fp64": errs,
            "mass_drift_rel": {"fp64": (c64.state_sums(s64)[0] - m64) / total,
                               "fp32": (c32.state_sums(s32)[0] - m32) / total},
            "bad_cells": {"fp64": c64.check_state(s64), "fp32": c32.check_state(s32)}}


ENS_SIZES = ((32, 32, 32), (64, 64, 32), (96, 96, 48), (128, 128, 64))


def ensemble_members(a):
    """The seeded members of the batching form: size picks, member configs and the
    init_state arguments of each member, drawn in member order."""
    import numpy as np
    from awflcloud_b200 import capi
    rng = np.random.default_rng(20261203)
    picks = rng.integers(0, len(ENS_SIZES), size=a.ens_members)
    cfgs = [dict(nx=ENS_SIZES[p][0], ny=ENS_SIZES[p][1], nz=ENS_SIZES[p][2], precision=capi.FP32, ord_=5)
            for p in picks]
    inits = []
    for i in range(len(cfgs)):
        r = float(rng.uniform(1000.0, 3000.0))
        inits.append(dict(kind=1, shape=1, x0=float(rng.uniform(5e3, 15e3)), y0=float(rng.uniform(5e3, 15e3)),
                          z0=float(rng.uniform(1.5e3, 3e3)), xrad=r, yrad=r, zrad=r, amp=float(rng.uniform(1, 4)),
                          pwr=1.0, noise_amp=0.01, noise_seed=20261203 + i))
    return picks, cfgs, inits


def ensemble_ranks_leg(a, local, rank, world):
    """The batching form over N GPUs: the one-GPU leg's seeded members spread over the ranks
    by cell count (awflcloud_b200.members), each rank's share one ensemble on its own GPU,
    no communication while stepping; the step loop timed on each rank's stream, maximum
    over ranks. Total work is fixed as N grows (strong scaling)."""
    import torch
    import torch.distributed as dist
    from awflcloud_b200.members import RankEnsemble, member_cells
    picks, cfgs, inits = ensemble_members(a)
    R = RankEnsemble(cfgs, rank, world, device=local)
    states = []
    for i in R.share:
        m = R.member(i)
        s = m.new_state()
        m.init_state(s, **inits[i])
        R.bind(i, s, m.cfl(s, 0.8))
        states.append(s)
    stream = torch.cuda.current_stream()
    R.tune(reps=3, stream=stream)
    R.step(2, stream=stream)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    R.step(a.ens_steps, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) if R.share else 0.0
    dist.barrier()
    max_ms = max_over_ranks(ms, world)
    cells = sum(member_cells(cfgs))
    finite = all(bool(torch.isfinite(s).all().item()) for s in states)
    R.close()
    return {"workload": "%d FP32 ord-5 members, %d steps, over %d GPUs" % (a.ens_members, a.ens_steps, world),
            "value": round(cells * a.ens_steps / (max_ms * 1e-3) / 1e6, 3), "unit": UNIT,
            "ms_per_step": round(max_ms / a.ens_steps, 4), "scaling": "strong",
            "cells_per_rank": [sum(member_cells([cfgs[i] for i in sh])) for sh in R.shares],
            "members_per_rank": [len(sh) for sh in R.shares],
            "parallelism": "members assigned to ranks by cell count (largest first onto the least-loaded "
                           "rank); one ensemble per GPU; no collective while stepping",
            "finite_on_rank0": finite}


def ensemble_leg(a, local):
    """Batching form: ens_members FP32 ord-5 members with seeded sizes from ENS_SIZES and
    seeded bubbles (centre x, y in [5, 15] km, z in [1.5, 3] km, amp in [1, 4] K, radius in
    [1, 3] km), advanced ens_steps steps by the ensemble (one persistent kernel per split
    stage, two steps per CUDA-graph replay, autotuned tile shapes), against the same
    members stepped one after another through awfl_step."""
    import numpy as np
    import torch
    from awflcloud_b200 import capi
    picks, cfgs, inits = ensemble_members(a)
    E = capi.Ensemble(cfgs, device=local)
    states, dts = [], []
    for i, m in enumerate(E.members):
        s = m.new_state()
        m.init_state(s, **inits[i])
        dt = m.cfl(s, 0.8)
        E.bind(i, s, dt)
        states.append(s)
        dts.append(dt)
    cells = sum(c["nx"] * c["ny"] * c["nz"] for c in cfgs)
    stream = torch.cuda.current_stream()
    table = E.tune(reps=3, stream=stream)
    E.step(2, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    E.step(a.ens_steps, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ens_ms = e0.elapsed_time(e1)
    # the same members, one context at a time (3 launches per member per step)
    for i, m in enumerate(E.members):
        m.step(states[i], dts[i])
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.ens_steps):
        for i, m in enumerate(E.members):
            m.step(states[i], dts[i])
    e1.record(stream)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    counts = {"%dx%dx%d" % s: int((picks == k).sum()) for k, s in enumerate(ENS_SIZES)}
    # load report: each size class alone, as an ensemble of its members and member by member
    by_size = []
    for k, size in enumerate(ENS_SIZES):
        idx = [i for i in range(len(cfgs)) if picks[i] == k]
        if not idx:
            continue
        sub = capi.Ensemble([cfgs[i] for i in idx], device=local)
        sub_states = [states[i].clone() for i in idx]
        for q, i in enumerate(idx):
            sub.bind(q, sub_states[q], dts[i])
        sub.tune(reps=3, stream=stream)
        sub.step(2, stream=stream)
        nst = 10
        torch.cuda.synchronize()
        e0.record(stream)
        sub.step(nst, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        sub_ms = e0.elapsed_time(e1)
        e0.record(stream)
        for _ in range(nst):
            for q, i in enumerate(idx):
                E.members[i].step(sub_states[q], dts[i])
        e1.record(stream)
        torch.cuda.synchronize()
        one_ms = e0.elapsed_time(e1)
        c_cells = len(idx) * size[0] * size[1] * size[2]
        by_size.append({"size": "%dx%dx%d" % size, "members": len(idx), "cells": c_cells,
                        "ensemble_value": round(c_cells * nst / (sub_ms * 1e-3) / 1e6, 1),
                        "sequential_value": round(c_cells * nst / (one_ms * 1e-3) / 1e6, 1)})
        del sub
    return {"workload": "%d FP32 ord-5 members, %d steps, sizes %s" % (a.ens_members, a.ens_steps, counts),
            "by_size": by_size,
            "value": round(cells * a.ens_steps / (ens_ms * 1e-3) / 1e6, 3), "unit": UNIT,
            "ms_per_step": round(ens_ms / a.ens_steps, 4),
            "sequential_value": round(cells * a.ens_steps / (seq_ms * 1e-3) / 1e6, 3),
            "speedup_vs_sequential": round(seq_ms / ens_ms, 3),
            "tuned_shapes": [{"dir": "xyz"[d], "chunk": E.shape(d)[1], "lines": E.shape(d)[2], "grid": E.shape(d)[3],
                              "candidates_ms": [[c, w, round(ms, 4)] for c, w, ms in table[d]]} for d in range(3)],
            "gpu_launches_per_step": 3, "finite": all(bool(torch.isfinite(s).all().item()) for s in states)}


def run_ours(a):
    import torch
    import torch.distributed as dist
    from awflcloud_b200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    main_prec = capi.FP32 if a.precision == "fp32" else capi.FP64
    main = time_form(a, main_prec, local, world, clocks=ClockSampler(local))
    other = time_form(a, capi.FP64, local, world) if (main_prec == capi.FP32 and not a.no_compare) else None
    e2e = None if a.no_e2e else e2e_leg(a, main, torch.cuda.current_stream(), world)
    # the precision-matched end-to-end figure: the FP64 path through the same C ABI calls
    e2e64 = None
    if other is not None and not a.no_e2e:
        e2e64 = e2e_leg(a, other, torch.cuda.current_stream(), world)
    # the batching form over the ranks (every rank takes part); on one GPU the leg below
    ens_ranks = ensemble_ranks_leg(a, local, rank, world) if (world > 1 and not a.no_ensemble) else None

    if rank == 0:
        line = {"metric": METRIC, "value": round(main["value"], 3), "unit": UNIT, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(main["ms_per_step"], 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if main_prec == capi.FP64 else "f32", "data": DATA,
                "config": bench_config(a),
                "parallelism": ("x slabs of one %dx%dx%d grid, %d cells wide per GPU; NCCL send/recv of "
                                "hs+1 halo columns per side before every x split, dt by all-reduce MIN"
                                % (a.nx * world, a.ny, a.nz, a.nx)) if world > 1 else "single GPU",
                "roofline": main["roofline"], "gpu_launches": (4 if world > 1 else 3) * a.steps, "finite": main["finite"],
                "clocks": main["clocks"], "flops_per_cell_step": main["flops"]}
        if other is not None:
            line["fp64"] = {"value": round(other["value"], 3), "ms_per_step": round(other["ms_per_step"], 4),
                            "roofline": other["roofline"], "finite": other["finite"]}
            if e2e64 is not None:
                line["fp64"]["e2e"] = e2e64
            line["fp32_over_fp64"] = round(main["value"] / other["value"], 3)
            errs = rel_l2_after(a, 100, local)
            line["rel_l2_vs_fp64_after_100_steps"] = {"rho": errs[0], "rho_u": errs[1], "rho_v": errs[2],
                                                      "rho_w": errs[3], "rho_theta": errs[4]}
        if e2e is not None:
            line["e2e"] = e2e
        line["output"] = output_leg(main["ctx"], main["state"])
        if not a.no_adjoint:
            line["adjoint"] = adjoint_leg(a, local)
        if ens_ranks is not None:
            line["ensemble"] = ens_ranks
        elif not a.no_ensemble:
            line["ensemble"] = ensemble_leg(a, local)
        if not a.no_precision:
            line["precision"] = precision_leg(a, local)
        if not a.no_ord9 and a.ord == 5:
            line["ord9"] = ord9_leg(a, local)
        if not a.no_tracers:
            line["tracers"] = tracers_leg(a, local)
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(a)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def e2e_leg(a, form, stream, world):
    """The same metric through the C ABI with HOST buffers: every step copies its input
    state from pinned host memory to the device, advances it one time step and copies the
    result back. Steps rotate over three device buffers on three streams, so that the
    host-to-device copies run back to back while earlier steps compute and copy their
    results back (the link is full duplex: 55-57 GB/s each way alone, ~92 GB/s both ways
    together on this box, which bounds a step at ~7.7 ms for 357 MB each way; two buffers
    gave 8.4 ms). The copies of every step stay inside the timed region."""
    import torch
    import torch.distributed as dist
    from awflcloud_b200 import capi
    L = capi.lib()
    ctx, st, dt, step = form["ctx"], form["state"], form["dt"], form["step"]
    nbytes = st.numel() * st.element_size()
    host_in = torch.empty_like(st, device="cpu").pin_memory()
    # N > 1: the slabs' column exchange orders its NCCL operations with one stream, so
    # the steps run on that one stream (no overlap of copies and compute across steps)
    nbuf = 3 if world == 1 else 1
    host_out = [torch.empty_like(st, device="cpu").pin_memory() for _ in range(nbuf)]
    host_in.copy_(st)
    dev = [st] + [torch.empty_like(st) for _ in range(nbuf - 1)]
    streams = [torch.cuda.Stream() for _ in range(nbuf)]

    def one(n):
        k = n % nbuf
        with torch.cuda.stream(streams[k]):
            s = streams[k].cuda_stream
            assert L.awfl_copy_h2d(dev[k].data_ptr(), host_in.data_ptr(), nbytes, s) == 0
            step(dev[k], dt)
            assert L.awfl_copy_d2h(host_out[k].data_ptr(), dev[k].data_ptr(), nbytes, s) == 0

    for s_ in streams:
        s_.wait_stream(stream)
    for n in range(nbuf):
        one(n)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s_ in streams:
        s_.wait_stream(stream)
    for n in range(a.steps):
        one(n)
    for s_ in streams:
        stream.wait_stream(s_)
    e1.record(stream)
    torch.cuda.synchronize()
    max_ms = max_over_ranks(e0.elapsed_time(e1), world)
    cells = a.nx * a.ny * a.nz
    return {"value": round(job_throughput(world, cells, a.steps, max_ms), 3), "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "path": "per step: awfl_copy_h2d + awfl_step + awfl_copy_d2h from/to pinned host buffers, "
                    "three device buffers on three streams (copies overlap compute and each other)"}


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.only:
        import torch
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        leg = {"adjoint": adjoint_leg, "ensemble": ensemble_leg, "precision": precision_leg,
               "ord9": ord9_leg, "tracers": tracers_leg}[a.only](a, local)
        print(json.dumps({"leg": a.only, **leg}))
        return 0
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
