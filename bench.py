"""Chemistry source-term benchmark: cells/s per flow step on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|small|large] [--cells n]

A step is one flow step of the chemistry source: every cell of the workload
is integrated over dt by the FP64 implicit-Euler integrator (one persistent
work-queue launch, cells ordered stiffest-first by the previous step's
Newton counts), timed as one replay of the captured flow step (CUDA graph:
queue reset, integrator launch, re-ordering). Each step starts from the same
seeded inputs, restored from a pristine device copy and followed by an L2
flush (a 256 MiB write) outside the per-step CUDA-event window. The kernel
is picked by the autotuner (openhurricane_b200/autotune.py) on a strided
sample of the workload's cells unless --kernel names one.

The timed steps are exactly --steps; the legs after them (end to end, the
CPU baseline, the gated surrogate: fixed sizes, 3 timed steps whatever
--steps says) run within --budget-s of wall-clock time, and a leg that would
overrun it is skipped and says so in the JSON line.

Workloads (seeded synthetic; no public dataset exists for this path):
  batched  9 species / 21 reactions, 1,048,576 cells, 20 % near ignition and
           80 % near equilibrium (chemical equilibrium at the cell's T and p,
           then T jittered by +-2 K), dt = 1e-5 s     (default)
  small    same mechanism, 4096 cells, Dirichlet states, dt = 1e-6 s
  large    53 species / 325 reactions, 262,144 cells, dt = 1e-6 s

Keys beyond the value: `e2e` is the same metric through hc_integrate_host
with pinned host buffers (copies in the timed region); `roofline` is the
integrator kernel's algorithmic FP64 FLOP rate (flop model of
openhurricane_b200/workloads.py times the Newton/Jacobian/LU counters) over
the FP64 FMA peak measured live by hc_probe_fp64_peak on this GPU;
`cpu_baseline` is the reference's own CPU integrator (oracle/_ref/hurchem_ref,
built from the reference sources) on a bounded sample of the same cells, one
process per host core.

--impl reference times that reference CPU path alone on the same workload,
config, metric and unit. With N > 1 ranks (torchrun), every rank integrates
its own replica of the workload (the path does not shard: replicas only);
the time is the max over ranks and the value counts all ranks' cells.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "chem cells/s per flow step, plain FP64 vs gated surrogate @ max|ΔT|<5K, 1 B200"
UNIT = "cells/s"
WORKLOAD_CELLS = {"batched": 1048576, "small": 4096, "large": 262144}
L2_FLUSH_BYTES = 256 << 20
SUR_STEPS = 3            # timed gated-surrogate steps (fixed, whatever --steps)
# DRAM bytes (read + write) per cell of one integrator launch on the 9-species
# mechanism: ncu dram__bytes_read.sum + dram__bytes_write.sum of
# integrate_w_kernel<10> over 37,888 batched cells (4.971776 + 2.029312 MB,
# profiles/integrator_warp_per_cell_batched.md), divided by the cells; the
# traffic grows with the cells integrated
DRAM_BYTES_PER_CELL = {9: (4.971776e6 + 2.029312e6) / 37888.0}


# ----------------------------------------------------------------------------- helpers
def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- time budget
def surrogate_leg_seconds(step_s: float, samples: int, ncells: int, epochs: int) -> float:
    """Estimated wall time of the gated-surrogate leg: sample generation (two
    FP64 integrations of `samples` cells: 0.74 plain steps for 524,288 samples
    on the 1,048,576-cell workload), training (13.4 s for 150 epochs of
    524,288 samples) and SUR_STEPS + 1 gated steps (0.41 of a plain step each
    at a 29 % reject rate), with margins. Its sizes are fixed: --steps does
    not enter."""
    return step_s * (1.5 * samples / ncells + 0.6 * (SUR_STEPS + 1)) + 3e-7 * epochs * samples


def fits_budget(elapsed_s: float, leg_s: float, budget_s: float, reserve_s: float = 60.0) -> bool:
    """A leg runs only if it ends `reserve_s` before the wall-clock budget."""
    return elapsed_s + leg_s <= budget_s - reserve_s


# ----------------------------------------------------------------------------- workloads
def build_workload(name: str, ncells: int, seed_offset: int):
    from openhurricane_b200 import workloads
    if name == "small":
        return workloads.make_small(ncells, seed=1001 + seed_offset)
    if name == "large":
        return workloads.make_large(ncells, seed=3003 + seed_offset)
    if name == "batched":
        return workloads.make_batched(ncells, seed=2002 + seed_offset)
    raise ValueError(f"unknown workload {name}")


def workload_config(wl, name: str) -> dict:
    return {"workload": f"{name}: {wl.tables.nsp} species / {wl.tables.nrc} reactions, "
                        f"{wl.n} cells, dt={wl.dt:g} s" + (f" ({wl.note})" if wl.note else ""),
            "species": int(wl.tables.nsp), "reactions": int(wl.tables.nrc), "cells": wl.n,
            "dt_s": wl.dt, "solver": "ImplicitEuler atol 1e-11 rtol 1e-4 maxstep 10000",
            "l2": "256 MiB L2 flush between timed steps"}


# ----------------------------------------------------------------------------- reference CPU
def reference_cpu(wl, target_seconds: float, cores: int, sample_offset: int = 0):
    """Time the reference's CPU integrator on a strided sample of the
    workload's cells. Returns (cells/s, sample cells, seconds, kind, note)."""
    from oracle import refrun
    from openhurricane_b200 import workloads
    if not refrun.available():
        return None
    work = tempfile.mkdtemp(prefix="hc_refbench_")
    case = os.path.join(work, "case.cont")
    refrun.write_case(case, *wl.files, dict(workloads.SOLVER_OPTS))
    n = wl.n
    # calibrate: one process on a handful of cells
    cal = np.arange(sample_offset % 16, n, max(1, n // 64))[:64]
    r = refrun.integrate(case, wl.T[cal], wl.p[cal], wl.rho[cal], wl.dt, wl.dt,
                         wl.Y[:, cal], procs=1, workdir=work)
    per_cell = max(r["seconds"], 1e-6) / cal.size
    m = int(min(n, max(cores, target_seconds * cores / per_cell)))
    stride = max(1, n // m)
    idx = np.arange(sample_offset % stride, n, stride)[:m]
    r = refrun.integrate(case, wl.T[idx], wl.p[idx], wl.rho[idx], wl.dt, wl.dt, wl.Y[:, idx],
                         procs=cores, workdir=work)
    secs = r["seconds"]
    return idx.size / secs, int(idx.size), secs


# ----------------------------------------------------------------------------- GPU arm
def tune_launch(mech, wl, dev):
    """The autotuner (openhurricane_b200/autotune.py) over the integrator
    kernels that take this mechanism, on a strided sample of the workload's
    cells with each cell's Newton iterations capped (equal work per cell, a
    fraction of a second per trial)."""
    import torch
    from openhurricane_b200 import _capi, autotune, workloads
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    m = min(wl.n, 16384)
    idx = np.linspace(0, wl.n - 1, m).astype(np.int64)
    o = _capi.default_opts(max_newton_total=400, **workloads.SOLVER_OPTS)
    dt = torch.full((m,), wl.dt, dtype=torch.float64, device=dev)
    r = autotune.autotune(mech, d(wl.T[idx]), d(wl.p[idx]), d(wl.rho[idx]), d(wl.Y[:, idx]), dt,
                          opts=o, sample=m, repeats=2)
    return {"kernel": r["kernel"], "block": r["block"], "source": "autotuner",
            "sample_cells": r["sample_cells"], "newton_cap_per_cell": 400,
            "trials": r["trials"]}


def run_ours(args, ws, rank, local):
    import torch
    import ctypes as C
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import ChemistrySource, Flow, Mechanism, integrate_host

    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    t_start = time.perf_counter()
    elapsed = lambda: time.perf_counter() - t_start
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)

    name = args.workload
    ncells = args.cells or WORKLOAD_CELLS[name]
    wl = build_workload(name, ncells, seed_offset=rank)
    mech = Mechanism(wl.tables)
    n, nsp = wl.n, wl.tables.nsp
    tuning = None
    if args.kernel is not None:
        mech.set_tuning(args.kernel, args.block)
        tuning = {"kernel": args.kernel, "block": args.block, "source": "--kernel"}
    else:
        tuning = tune_launch(mech, wl, dev)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    T0, p0, rho0, Y0 = d(wl.T), d(wl.p), d(wl.rho), d(wl.Y)
    flow = Flow(T0.clone(), p0, rho0.clone(), Y0.clone())
    cs = ChemistrySource(mech, flow, **workloads.SOLVER_OPTS)
    dt = torch.full((n,), wl.dt, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def restore():
        flow.T.copy_(T0)
        flow.rho.copy_(rho0)
        flow.Y.copy_(Y0)
        if cs.dtInit is not None:
            cs.dtInit.copy_(dt)     # in place: a captured step reads this buffer

    # warm-up: the first call also fixes the stiffness order for later steps
    counters = None
    t_w = time.perf_counter()
    for w in range(args.warmup):
        restore()
        cs.solveUpdate(dt, 1.0, counters=(w == args.warmup - 1))
    torch.cuda.synchronize()
    warm_s = (time.perf_counter() - t_w) / args.warmup
    counters = dict(cs.last_counters)
    # the timed step is one replay of the captured flow step (queue reset,
    # integrator launch, stiffness re-ordering)
    graph = cs.capture_update(dt, 1.0) if args.graph else None

    fm = workloads.flop_model(wl.tables)
    flops_per_launch = workloads.work_flops(counters, fm)

    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        restore()
        flush.fill_(float(k))
        ev[k][0].record(stream)
        if graph is not None:
            graph.replay()
        else:
            cs.solveUpdate(dt, 1.0)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms_local = float(sum(step_ms))

    lib = _capi.load()
    # a step is one integrator launch plus the stiffness re-ordering of the
    # cells (an argsort of the per-cell Newton counts, a negligible part of
    # the step): the step time is the kernel time of the roofline
    kernel_ms = ms_local / args.steps
    clk = clocks.stop()
    # the FP64 result of the last timed step (from the pristine inputs): the
    # reference the surrogate is compared with
    fp64_ref = (flow.T.clone(), flow.Y.clone())

    # end to end: host (pinned) buffers through hc_integrate_host
    pin = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64).pin_memory()
    hT0, hrho0, hY0 = wl.T.copy(), wl.rho.copy(), np.ascontiguousarray(wl.Y)
    hT, hp, hrho, hY = pin(wl.T), pin(wl.p), pin(wl.rho), pin(wl.Y)
    hdt, hsub = pin(np.full(n, wl.dt)), pin(np.full(n, wl.dt))
    hst = torch.zeros(n, dtype=torch.int32).pin_memory()
    vp = lambda t: C.c_void_p(t.data_ptr())
    e2e_steps = max(1, args.e2e_steps)

    def host_call():
        o = cs.opts
        r = lib.hc_integrate_host(mech.handle, C.byref(o), n, vp(hT), vp(hp), vp(hrho), vp(hY),
                                  vp(hdt), 1.0, vp(hsub), None, vp(hst), None,
                                  C.c_void_p(stream.cuda_stream))
        _capi.check(r, "hc_integrate_host")

    def host_restore():
        hT.numpy()[:] = hT0
        hrho.numpy()[:] = hrho0
        hY.numpy()[:] = hY0
        hsub.numpy()[:] = wl.dt

    host_restore()
    host_call()
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for k in range(e2e_steps):
        host_restore()
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        host_call()
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms += a.elapsed_time(b)
    e2e_ms /= e2e_steps
    h2d = n * (5 + nsp) * 8
    d2h = n * (3 + nsp) * 8 + n * 4

    step_s = ms_local / args.steps * 1e-3
    sur = None
    if args.surrogate and name == "batched":
        est = surrogate_leg_seconds(step_s, args.sur_samples, n, args.sur_epochs)
        if not fits_budget(elapsed(), est, args.budget_s):
            sur = {"skipped": f"wall-clock budget: needs about {est:.0f} s, "
                              f"{args.budget_s - elapsed():.0f} s left of --budget-s {args.budget_s:g}"}
    if args.surrogate and name == "batched" and sur is None:
        sur = surrogate_leg(args, wl, mech, (T0, p0, rho0, Y0), dt, fp64_ref,
                            ms_local / args.steps, flush, rank, counters["n_newton"])
    if graph is not None:
        del graph

    props = None
    if name == "large":
        props = properties_leg(mech, (T0, p0, rho0, Y0), flush, args.prop_cells)

    # FP64 peak on this GPU
    peak = C.c_double(0.0)
    _capi.check(lib.hc_probe_fp64_peak(1 << 16, C.byref(peak), C.c_void_p(stream.cuda_stream)),
                "hc_probe_fp64_peak")

    from openhurricane_b200 import replicas
    ms_total, e2e_ms = replicas.max_over_ranks([ms_local, e2e_ms], device=dev)
    cells_all = replicas.sum_over_ranks([n], device=dev)[0]
    ms_step = ms_total / args.steps
    value = replicas.whole_job_rate([cells_all], ms_step)

    out = None
    if rank == 0:
        achieved = flops_per_launch / (kernel_ms * 1e-3) / 1e12
        cores = _host_cores()
        cpu = None
        if not args.no_cpu_baseline:
            cpu_s = max(2.0, min(args.cpu_seconds, args.budget_s - elapsed() - 30.0))
            cb = reference_cpu(wl, cpu_s, cores)
            if cb is not None:
                v, m, secs = cb
                cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                       "sample": f"{m} of {n} cells (strided), reference ImplicitEuler, "
                                 f"{cores} single-threaded processes, {secs:.1f} s"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)", "impl": "ours",
            "config": dict(workload_config(wl, name), parallelism=f"replicas x{ws}"),
            "e2e": {"value": replicas.whole_job_rate([cells_all], e2e_ms), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak.value,
                         "unit": "TFLOP/s", "frac": achieved / peak.value,
                         "traffic": (DRAM_BYTES_PER_CELL[nsp] * n if nsp in DRAM_BYTES_PER_CELL
                                     else None),
                         "traffic_note": "DRAM bytes per launch, scaled from an ncu capture "
                                         "of the warp-per-cell kernel on 37,888 cells by the "
                                         "cell count",
                         "peak_source": "FP64 FMA probe measured in this run "
                                        "(no FP64 figure in the measured peaks file)",
                         "kernel_ms": kernel_ms, "flops_per_launch": flops_per_launch},
            "counters": counters,
            "tuning": tuning,
            "wall_s": {"warmup_step": warm_s, "run_so_far": elapsed()},
            "clocks": clk,
            "cpu_baseline": cpu,
            "surrogate": sur,
            "properties": props,
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def hbm_peak_gbs():
    """Measured HBM copy bandwidth of this pool's B200s, else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def properties_leg(mech, fields0, flush, prop_cells):
    """Mixture properties (h_i, cp, mu, kappa, D_i) of the workload's cells
    tiled to prop_cells cells: one properties_kernel launch, timed with CUDA
    events after an L2 flush; algorithmic bytes = inputs T, p, Y and outputs
    h_i, D_i, cp, mu, kappa (8 B each)."""
    import torch
    T0, p0, _, Y0 = fields0
    n0 = int(T0.shape[0])
    reps = max(1, prop_cells // n0)
    T = T0.repeat(reps).contiguous()
    p = p0.repeat(reps).contiguous()
    Y = Y0.repeat(1, reps).contiguous()
    n, nsp = int(T.shape[0]), int(Y.shape[0])
    stream = torch.cuda.current_stream()
    for _ in range(3):
        mech.properties(T, p, Y)
    times = []
    for k in range(5):
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        mech.properties(T, p, Y)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms = float(np.median(times))
    nbytes = n * 8.0 * ((2 + nsp) + (2 * nsp + 3))
    peak, src = hbm_peak_gbs()
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"cells": n, "ms": ms, "cells_per_s": n / (ms * 1e-3), "bound": "hbm",
            "achieved_GBs": gbs, "peak_GBs": peak, "peak_source": src, "frac": gbs / peak,
            "bytes_per_launch": nbytes}


def surrogate_leg(args, wl, mech, fields0, dt, fp64_ref, plain_ms, flush, rank, plain_newton):
    """Train the gated surrogate on samples of the FP64 GPU integrator (states
    of the same distribution, another seed), then time its flow step on the
    workload's cells and compare it with the FP64 step."""
    import torch
    from openhurricane_b200 import _capi, workloads
    from openhurricane_b200.chemistry import Flow
    from openhurricane_b200.surrogate import Surrogate, generate_samples, integrate_device
    dev = fields0[0].device
    opts = _capi.default_opts(**workloads.SOLVER_OPTS)
    t0 = time.perf_counter()

    base = workloads.make_batched(65536, seed=5005 + rank)
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    smp = generate_samples(mech, d(base.T), d(base.p), d(base.rho), d(base.Y), wl.dt,
                           args.sur_samples, seed=11 + rank, opts=opts)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    sur = Surrogate(mech, n_hidden=3, width=256, max_batch=65536, seed=3 + rank, n_ensemble=3)
    sur.fit_normalisation(smp["T"], smp["p"], smp["Y"], smp["dt"], smp["dT"], smp["dY"])
    X = sur.features(smp["T"], smp["p"], smp["Y"], smp["dt"])
    D = sur.targets(smp["dT"], smp["dY"])
    n_train = int(X.shape[0])
    del smp
    t1 = time.perf_counter()
    losses = sur.train(X, D, epochs=args.sur_epochs, batch=8192, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    del X, D
    T0, p0, rho0, Y0 = fields0
    n = int(T0.shape[0])
    flow = Flow(T0.clone(), p0, rho0.clone(), Y0.clone())
    stream = torch.cuda.current_stream()

    def restore():
        flow.T.copy_(T0)
        flow.rho.copy_(rho0)
        flow.Y.copy_(Y0)

    restore()
    sur.step(flow, dt, opts=opts)     # warm-up
    ms, rej = [], []
    for k in range(SUR_STEPS):
        restore()
        flush.fill_(float(k))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fb = {}
        nr, accept = sur.step(flow, dt, opts=opts, counters=fb)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
        rej.append(nr)
    Tref, Yref = fp64_ref
    acc = accept.bool()
    dT = (flow.T - Tref).abs()
    dY = (flow.Y - Yref).abs()
    A = torch.tensor(wl.tables.elem_matrix / wl.tables.W[None, :], dtype=torch.float64, device=dev)
    e0, e1 = A @ Y0, A @ flow.Y
    rel = ((e1 - e0).abs() / e0.abs().max(dim=0, keepdim=True).values)
    sur_ms = float(np.mean(ms))
    return {"cells_per_s": n / (sur_ms * 1e-3), "ms_per_step": sur_ms,
            "speedup_vs_plain": plain_ms / sur_ms,
            "reject_rate": float(np.mean(rej)) / n,
            "fp64_work_gain": plain_newton / max(1, fb.get("n_newton", 0)),
            "fp64_work_gain_note": "Newton iterations of the plain step / of the gated step's FP64 "
                                   "fallback on the same cells",
            "max_abs_dT_K": float(dT.max()), "max_abs_dT_accepted_K": float(dT[acc].max()) if
            bool(acc.any()) else 0.0,
            "linf_dY": float(dY.max()),
            "max_element_rel_err_accepted": float(rel[:, acc].max()) if bool(acc.any()) else 0.0,
            "network": "12 -> 3 x 256 GELU -> 10 (x3 ensemble), BF16 tcgen05 / FP32 accumulate",
            "gate": {"tol_T_K": sur.gate.tol_T, "spread_T_K": sur.spread_T,
                     "spread_Y": sur.spread_Y, "y_neg": sur.gate.y_neg},
            "train_samples": n_train, "train_epochs": args.sur_epochs, "batch": 8192,
            "final_loss": losses[-1] if losses else None,
            "sample_gen_s": t_gen, "train_s": t_train,
            "compared_with": "FP64 GPU integrator on the same cells (atol 1e-11, rtol 1e-4)"}


def run_reference(args, ws, rank):
    """Reference CPU integrator on the host cores; rank 0 only."""
    if rank != 0:
        return None
    from oracle import refrun
    from openhurricane_b200 import workloads
    name = args.workload
    ncells = args.cells or WORKLOAD_CELLS[name]
    if not refrun.available():
        return {"impl": "reference", "unavailable": "reference CPU binary oracle/_ref/hurchem_ref "
                                                    "not built (make -f oracle/Makefile.ref)"}
    cores = _host_cores()
    if name == "batched":
        wl = workloads.make_batched(ncells, seed=2002)
    elif name == "small":
        wl = workloads.make_small(ncells)
    else:
        wl = workloads.make_large(ncells)
    budget = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for w in range(args.warmup):
        reference_cpu(wl, min(budget, 2.0), cores, sample_offset=w)
    vals, cells, secs = [], 0, 0.0
    for k in range(args.steps):
        v, m, s = reference_cpu(wl, budget, cores, sample_offset=args.warmup + k)
        vals.append(v)
        cells += m
        secs += s
    value = cells / secs
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "impl": "reference",
        "config": dict(workload_config(wl, name), parallelism="host cores"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"each step a strided sample of ~{cells // args.steps} of "
                                   f"{wl.n} cells, {cores} single-threaded processes"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }


# ----------------------------------------------------------------------------- profiling cases
def run_profile(args):
    """One small, fixed piece of work for an ncu capture or a quick timing
    (no JSON bench line): `integrate` one hc_integrate launch of --cells
    seeded cells of --workload (strided from its cell set) with a per-cell
    Newton cap --cap (0: none) and --kernel / --block; `gemm` the surrogate's
    BF16 tcgen05 GEMM on --gemm M,N,K (three untimed launches, ten timed);
    `props` the mixture-property kernel on --cells cells of the 53-species
    workload (three untimed launches, five timed after a 256 MiB L2 flush)."""
    import ctypes as C
    import torch
    from openhurricane_b200 import _capi, synth, workloads
    from openhurricane_b200.chemistry import Mechanism
    dev = torch.device("cuda:0")
    d = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()

    def timed(fn, reps, flush=None):
        for _ in range(3):
            fn()
        times = []
        for k in range(reps):
            if flush is not None:
                flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            fn()
            b.record(st)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        return float(np.median(times))

    if args.profile == "gemm":
        from openhurricane_b200.surrogate import gemm_bf16
        M, N, K = (int(x) for x in args.gemm.split(","))
        g = torch.Generator(device="cpu").manual_seed(0)
        A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(dev)
        B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(dev)
        ms = timed(lambda: gemm_bf16(A, B), 10)
        return {"profile": "gemm", "M": M, "N": N, "K": K, "ms": ms,
                "TFLOPs": 2.0 * M * N * K / (ms * 1e-3) / 1e12}
    if args.profile == "props":
        n = args.cells or 262144
        _, _, t = workloads.mechanism_files("large")
        c = workloads.large_cells(n, 3003)
        m = Mechanism(t)
        T, p, Y = d(c.T), d(c.p), d(c.Y)
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
        ms = timed(lambda: m.properties(T, p, Y), 5, flush)
        nbytes = n * 8.0 * ((2 + t.nsp) + (2 * t.nsp + 3))
        return {"profile": "props", "cells": n, "species": t.nsp, "ms": ms,
                "cells_per_s": n / (ms * 1e-3), "algorithmic_bytes": nbytes,
                "GB_per_s": nbytes / (ms * 1e-3) / 1e9}
    # integrate
    n = args.cells or 4096
    name = args.workload
    if name == "batched":
        wl = workloads.make_batched(max(n, 65536), pool=512)
        idx = np.linspace(0, wl.n - 1, n).astype(np.int64)
        T0, p0, r0, Y0, dt = wl.T[idx], wl.p[idx], wl.rho[idx], wl.Y[:, idx], wl.dt
        t = wl.tables
    else:
        _, _, t = workloads.mechanism_files(name)
        c = workloads.small_cells(n, 1001) if name == "small" else workloads.large_cells(n, 3003)
        T0, p0, r0, Y0, dt = c.T, c.p, synth.mixture_density(t.W, c), c.Y, args.dt
    m = Mechanism(t)
    if args.kernel is not None:
        m.set_tuning(args.kernel, args.block)
    T, p, rho, Y = d(T0), d(p0), d(r0), d(Y0)
    dtt = torch.full((n,), dt, dtype=torch.float64, device=dev)
    sub = dtt.clone()
    o = _capi.default_opts(max_newton_total=args.cap, **workloads.SOLVER_OPTS)
    vp = lambda x: C.c_void_p(x.data_ptr())
    cnt = _capi.HcCounters()
    t0 = time.perf_counter()
    rc = _capi.load().hc_integrate(m.handle, C.byref(o), n, vp(T), vp(p), vp(rho), vp(Y), vp(dtt),
                                   1.0, vp(sub), None, None, C.addressof(cnt),
                                   C.c_void_p(st.cuda_stream))
    _capi.check(rc, "hc_integrate")
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    return {"profile": "integrate", "workload": name, "cells": n, "cap": args.cap,
            "kernel": args.kernel, "seconds": secs, "newton": int(cnt.n_newton),
            "newton_per_s": cnt.n_newton / secs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOAD_CELLS), default="batched")
    ap.add_argument("--cells", type=int, default=0)
    ap.add_argument("--kernel", type=int, default=None, help="0 auto, 1 thread/cell, 2 group")
    ap.add_argument("--block", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--graph", type=int, default=1,
                    help="1: time each step as a replay of the captured flow step (CUDA graph)")
    ap.add_argument("--budget-s", type=float, default=1500.0,
                    help="wall-clock budget of the run: legs after the timed steps that would "
                         "overrun it are skipped (the timed steps never are)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--prop-cells", type=int, default=262144,
                    help="cells of the property leg (large workload)")
    ap.add_argument("--surrogate", type=int, default=1,
                    help="1: also train and time the gated surrogate (batched workload)")
    ap.add_argument("--sur-samples", type=int, default=524288)
    ap.add_argument("--sur-epochs", type=int, default=150)
    ap.add_argument("--profile", choices=["integrate", "gemm", "props"], default=None,
                    help="run one small profiling case instead of the benchmark")
    ap.add_argument("--cap", type=int, default=0, help="--profile integrate: Newton cap per cell")
    ap.add_argument("--dt", type=float, default=1e-6, help="--profile integrate: dt (small / large)")
    ap.add_argument("--gemm", default="8192,256,256", help="--profile gemm: M,N,K")
    args = ap.parse_args()
    if args.profile:
        print(json.dumps(run_profile(args)), flush=True)
        return
    if args.warmup < 1:
        raise SystemExit("--warmup must be >= 1")
    ws, rank, local = _dist()
    if args.impl == "reference":
        out = run_reference(args, ws, rank)
    else:
        out = run_ours(args, ws, rank, local)
    if out is not None and rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
