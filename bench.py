#!/usr/bin/env python
"""Benchmark of the ADER-DG hot path on B200.

Workload: 3D compressible Euler, ADER-DG order N=5 (6^3 Gauss-Legendre nodes
per cell), uniform 27^3 cells on the periodic unit cube, four seeded Gaussian
density pulses on rho = 1, one seeded velocity, p = 1 (seed 0). One bench step
is one non-fused ADER-DG time step over the whole mesh: Rusanov fluxes on all
faces, surface integral + solution update + admissible step (min-reduced on
the device), space-time predictor + volume integral with the new step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Under torchrun every rank runs an independent
replica of the workload (the solver is single-GPU; replicas only).
Metric: DoF-updates/s, one DoF-update = one (cell, node, conserved variable)
advanced by one step (ncells * 216 * 5 per step).

Besides the headline line's own keys, "limiter" reports the a-posteriori
limiter workload measured in the same run: 2D Euler N=5 circular explosion on
81x81 outflow cells, 11x11 MUSCL-Hancock subcells, DMP delta0 1e-4 and
epsilon 1e-3, run to t = 0.2 (--workload limiter prints it as its own line).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

# every mesh of the serving workload has its own stream: let CUDA map up to 32
# of them to separate hardware queues (the default 8 makes unrelated streams
# queue behind each other); read when the CUDA context is created
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

DIM, ORDER, CELLS, SEED = 3, 5, (27, 27, 27), 0
NVAR = 5
WORKLOAD = "euler3d_N5_27^3_periodic_4pulses"
METRIC = "ADER-DG DoF-updates/s on 1 B200, mixed vs FP64 at \u22641e-9 L2; p99 solve latency"
LIM_DIM, LIM_ORDER, LIM_CELLS, LIM_TEND = 2, 5, (81, 81), 0.2
# linear-kernel workload: elastic waves, 9 variables + 3 material parameters
EL_DIM, EL_ORDER, EL_CELLS, EL_NVAR, EL_NDATA = 3, 5, (27, 27, 27), 9, 12
EL_WORKLOAD = "elastic3d_N5_27^3_periodic_pulse_linear"
LIM_WORKLOAD = "euler2d_N5_81^2_explosion_limiter_outflow_t0.2"
# per-launch DRAM traffic of the predictor from the committed ncu capture
PROFILE_PREDICTOR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                                 "predictor_euler3d_N5_27cubed.md")


def dof_per_step():
    return int(np.prod(CELLS)) * (ORDER + 1) ** DIM * NVAR


def flux_flops(dim):
    # Euler flux at one node (pde.cuh EulerPDE::flux): 1/rho, |j|^2, p, (E+p)/rho,
    # and per direction 1 + 3*2 (+1 on the diagonal) + 1 products/sums
    return 1 + 5 + 4 + 2 + dim * 9


def predictor_flops(dim, N, sweeps, ncells, nV=NVAR, first_sweep_once=False, even_odd=False):
    """Algorithmic FLOPs of spaceTimePredictor + volumeIntegral (padding and
    idle lanes not counted): per Picard sweep per cell
    2 d nV b^(d+2) (derivatives) + 2 nV b^(d+2) (iK1) + 2 nV b^(d+1) (rhs0)
    + b^(d+1) flux evaluations; per cell once: time averaging +
    extrapolation 2(d+2) nV b^(d+1) + 8 d nV b^d, volume integral 2 d nV b^(d+1).
    `sweeps` is the total over all cells. With first_sweep_once the count is
    of the work the line-form kernel executes: every cell's first sweep
    starts from the time-constant guess, so its fluxes and derivative
    contractions are formed once instead of once per time slice (1/b). With
    even_odd (b even) each line contraction is the line-form kernel's split
    into even and odd parts, b^2 + 2 b instead of 2 b^2 flops per line."""
    b = N + 1
    per_line = b * b + 2 * b if (even_odd and b % 2 == 0) else 2 * b * b
    deriv = dim * nV * b ** dim * per_line + b ** (dim + 1) * flux_flops(dim)
    per_sweep = deriv + 2 * nV * b ** (dim + 2) + 2 * nV * b ** (dim + 1)
    per_cell = 2 * (dim + 2) * nV * b ** (dim + 1) + 8 * dim * nV * b ** dim + 2 * dim * nV * b ** (dim + 1)
    saved = deriv * (b - 1) / b * ncells if first_sweep_once else 0.0
    return per_sweep * sweeps + per_cell * ncells - saved


def bytes_per_step(dim, N, ncells, nV=NVAR, nD=NVAR):
    """compulsory HBM bytes of each phase per step (FP64)"""
    b = N + 1
    P, F = b ** dim, b ** (dim - 1)
    pred = 8 * ncells * (P * nD + 2 * dim * F * (nD + nV) + P * nV)
    riem = 8 * ncells * dim * (2 * F * nD + 4 * F * nV)
    corr = 8 * ncells * (2 * P * nD + P * nV + 2 * dim * F * nV)
    return dict(predictor=pred, riemann=riem, corrector=corr)


def linear_predictor_flops(dim, N, ncells, nV=EL_NVAR, nD=EL_NDATA):
    """Algorithmic FLOPs of the linear predictor (Cauchy-Kovalevski) + volume
    integral per launch: per derivative level (b of them) 2 b^(d+1) per
    gradient component the elastic product reads (6 of the 9 variables per
    direction) + per node the product (3 per direction: 2 for the moduli, 9
    products) and the level update and both time averages
    (d nV + 2 nV + 2 d nV); per cell once the boundary extrapolation
    4 d b^(d-1) b (nD + nV) and the volume integral 2 d nV b^d."""
    b = N + 1
    P = b ** dim
    used = 6 * dim  # gradient components the elastic non-conservative product reads
    per_level = 2 * used * b ** (dim + 1) + P * (dim * (2 + nV) + dim * nV + 2 * nV + 2 * dim * nV)
    per_cell = b * per_level + 4 * dim * b ** (dim - 1) * b * (nD + nV) + 2 * dim * nV * P
    return per_cell * ncells


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return dict(hbm_gbs=j.get("hbm_gbs", 6650.0), src="measured")
    return dict(hbm_gbs=6650.0, src="fallback")


class ClockSampler:
    """nvidia-smi samples during the timed region (median SM clock, reasons)."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return dict(sm_mhz=float(np.median(sm)), sm_max_mhz=mx, reasons=sorted(reasons), samples=len(sm))


PREDICTOR_SOURCES = ("exahype_b200/csrc/predictor_lines.cuh", "exahype_b200/csrc/aderdg.cuh",
                     "exahype_b200/csrc/pde.cuh", "exahype_b200/csrc/common.cuh", "exahype_b200/csrc/tmem.cuh")


def predictor_source_hash():
    """sha256 (first 16 hex digits) over the predictor kernel's sources"""
    import hashlib
    h = hashlib.sha256()
    for f in PREDICTOR_SOURCES:
        with open(os.path.join(REPO, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def predictor_traffic_bytes(variant):
    """(dram__bytes_read.sum + dram__bytes_write.sum of one predictor launch on
    the 27^3 N=5 mesh, source note) from the committed ncu summary's lines
    'traffic_bytes_per_launch: <n>', 'captured_variant: <v>' and
    'source_sha16: <hash of the kernel sources it was captured from>'. The
    figure is only used while the sources still hash the same and the run
    uses the captured variant; otherwise (None, why)."""
    rel = os.path.relpath(PROFILE_PREDICTOR, REPO)
    val, sha, var = None, None, None
    try:
        with open(PROFILE_PREDICTOR) as f:
            for line in f:
                t = line.strip()
                if t.startswith("traffic_bytes_per_launch:"):
                    val = float(t.split(":", 1)[1].strip().split()[0])
                elif t.startswith("source_sha16:"):
                    sha = t.split(":", 1)[1].strip().split()[0]
                elif t.startswith("captured_variant:"):
                    var = int(t.split(":", 1)[1].strip().split()[0])
    except OSError:
        return None, "no ncu summary at %s" % rel
    cur = predictor_source_hash()
    if val is None or sha != cur:
        return None, "%s was captured from other kernel sources (sha16 %s, now %s): traffic not reused" % (
            rel, sha, cur)
    if var != variant:
        return None, "%s was captured for predictor variant %s, this run uses %d: traffic not reused" % (
            rel, var, variant)
    return val, "%s (ncu capture of the same kernel sources and variant, sha16 %s)" % (rel, cur)


def reduce_max(x, world, device=None):
    """max over ranks of a scalar (identity for one rank)"""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_build(fast=True):
    """('ref_fast', description) for the timed -O3 build of the reference
    kernels when this CPU can run one, else ('ref', description of the
    parity build)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle
    if fast:
        path, name = pyoracle.fast_build(DIM)
        if path:
            return "ref_fast", "reference kernels built -O3 -march=%s (FMA contraction on)" % name
    return "ref", "reference kernels, parity build (-O2 -ffp-contract=off)"


def cpu_reference_run(steps, warmup, nthreads, cells=CELLS, runs=1, fast=True):
    """The reference's own generic kernels (compiled from its sources into
    oracle/_ref) driven by the oracle harness on the host cores: `warmup`
    steps, then `runs` timed runs of `steps` steps each (continuing the same
    run); the value is from the median run."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle
    from exahype_b200 import problems
    if not pyoracle.ref_available(DIM):
        return None
    impl, build = ref_build(fast)
    u, _ = problems.gaussian_pulses_3d(ORDER, cells, seed=SEED)
    m = pyoracle.Mesh(DIM, ORDER, cells, [1.0] * DIM, -1, impl=impl, nthreads=nthreads)
    m.set_solution(u)
    m.init(0.0)
    if warmup:
        m.step(warmup)
    times = []
    for _ in range(max(1, runs)):
        t0 = time.perf_counter()
        m.step(steps)
        times.append(time.perf_counter() - t0)
    el = float(np.median(times))
    dof = int(np.prod(cells)) * (ORDER + 1) ** DIM * NVAR * steps
    return dict(value=dof / el, seconds=el, run_seconds=times, steps=steps, cells=list(cells), build=build,
                cpu=cpu_model())


def run_reference_arm(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    nthreads = os.cpu_count() or 1
    runs = 5
    r = cpu_reference_run(a.steps, a.warmup, nthreads, runs=runs)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference kernels built from the "
                          "reference sources) is not present in this tree"}))
        return 0
    # the parity build (what the tests compare against), one run, for comparison
    rp = cpu_reference_run(a.steps, 0, nthreads, runs=1, fast=False) if r["build"].find("-O3") >= 0 else None
    ms = 1000.0 * r["seconds"] / a.steps
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "DoF-updates/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian pulses)",
        "config": {"workload": WORKLOAD, "dim": DIM, "order": ORDER, "cells": list(CELLS),
                   "dof_per_step": dof_per_step(), "l2": "inputs larger than L2 (170 MB solution)"},
        "cpu_baseline": {"value": r["value"], "unit": "DoF-updates/s", "cores": nthreads, "kind": "reference",
                         "cpu": r["cpu"], "build": r["build"],
                         "sample": "median of %d runs of %d full time steps of the 27^3 mesh after %d warm-up steps"
                                   " (run times %s s)" % (runs, a.steps, a.warmup,
                                                          ", ".join("%.2f" % x for x in r["run_seconds"]))},
        "e2e": {"value": r["value"], "unit": "DoF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if rp is not None:
        line["parity_build"] = {"value": rp["value"], "unit": "DoF-updates/s", "build": rp["build"],
                                "sample": "1 run of %d steps" % a.steps}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(a):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    import exahype_b200 as eb
    from exahype_b200 import problems

    u0, _ = problems.gaussian_pulses_3d(ORDER, CELLS, seed=SEED + rank)
    s = eb.Solver(DIM, ORDER, eb.PDE_EULER)
    if a.variant is not None:
        s.variant = a.variant  # also for the initial predictor
    m = eb.Mesh(s, CELLS, [0.0] * DIM, [1.0] * DIM, eb.BC_PERIODIC)
    m.set_solution(u0)
    m.init(0.0)
    stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
    if a.variant is None:
        # predictor shape chosen on the workload itself: one timed mesh step
        # per FP64 variant (after one untimed), before the warm-up steps
        vms = {}
        for v in (0, 1, 2, 3, 6, 7, 8):
            s.variant = v
            m.step(1)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            m.step(1)
            t1.record(stream)
            t1.synchronize()
            vms[v] = reduce_max(t0.elapsed_time(t1), world, dev)
        chosen = min(vms, key=vms.get)
        s.variant = chosen
        tune = {"chosen": chosen, "variant_ms_mesh_step": vms}
    else:
        s.variant = a.variant
        tune = {"chosen": a.variant, "forced": True}

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    # warm-up
    m.step(a.warmup)
    m.synchronize()
    st0 = m.state()
    m.phase_times(reset=True)
    m.set_profiling(True)
    clk = ClockSampler(local)
    barrier()
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(a.steps)
    e1.record(stream)
    e1.synchronize()
    barrier()
    clocks = clk.stop()
    m.set_profiling(False)
    ms_total = e0.elapsed_time(e1)
    ph = m.phase_times(reset=True)
    st1 = m.state()
    sweeps = st1["picard_sweeps"] - st0["picard_sweeps"]
    ms_total = reduce_max(ms_total, world, dev)
    dof = dof_per_step() * a.steps * world
    value = dof / (ms_total / 1000.0)

    # roofline of the dominant kernel (predictor + volume integral, FP64 pipe)
    ncells = int(np.prod(CELLS))
    pred_ms = ph["predictor"][0] / a.steps
    line_form = s.variant in (1, 2, 4, 5, 6, 7, 8)  # the line-form kernels form the first sweep once
    # algorithmic flops: the reference's loops (spaceTimePredictorNonlinear +
    # volumeIntegralNonlinear) for the sweeps the run took; executed: what the
    # chosen kernel does (first sweep once per cell, even/odd contractions)
    pflops = predictor_flops(DIM, ORDER, sweeps / a.steps, ncells)
    pflops_exec = predictor_flops(DIM, ORDER, sweeps / a.steps, ncells, first_sweep_once=line_form,
                                  even_odd=line_form and s.variant not in (4, 5))
    fp64_peaks = measure_fp64_peak() if not a.no_fp64_probe else None
    fp64_peak = max(fp64_peaks.values()) if fp64_peaks else None
    peaks = load_peaks()
    byt = bytes_per_step(DIM, ORDER, ncells)
    kernels = {}
    for name, bound in (("predictor", "fp64"), ("riemann", "hbm"), ("corrector", "hbm")):
        t_ms = ph[name][0] / a.steps
        if bound == "fp64":
            ach = pflops / (t_ms / 1e3) / 1e12
            kernels[name] = dict(bound="fp64", achieved=ach, unit="TFLOP/s", ms=t_ms,
                                 peak=fp64_peak, frac=(ach / fp64_peak) if fp64_peak else None)
        else:
            ach = byt[name] / (t_ms / 1e3) / 1e9
            kernels[name] = dict(bound="hbm", achieved=ach, unit="GB/s", ms=t_ms, peak=peaks["hbm_gbs"],
                                 frac=ach / peaks["hbm_gbs"])
    roof = dict(kernels["predictor"])
    traffic, tsrc = predictor_traffic_bytes(s.variant)
    roof.update(traffic=traffic, traffic_source=tsrc,
                peak_source="the larger of the FP64 DFMA and DMMA (mma.sync m8n8k4 f64) probes measured in this run "
                            "(%s TFLOP/s); MEASURED_PEAKS.json has no FP64 figure" % (
                                ", ".join("%s %.2f" % kv for kv in sorted((fp64_peaks or {}).items())) or "none"),
                algorithmic_flops_per_launch=pflops, executed_flops_per_launch=pflops_exec,
                executed_achieved=pflops_exec / (roof["ms"] / 1e3) / 1e12,
                executed_frac=(pflops_exec / (roof["ms"] / 1e3) / 1e12 / fp64_peak) if fp64_peak else None,
                flops_note="achieved counts the algorithm's flops, the reference's loops for the Picard sweeps the "
                           "run took (the work a launch completes); executed_* count what the chosen kernel "
                           "performs: the first sweep's fluxes and derivative contractions once per cell instead "
                           "of once per time slice, and each line contraction split into its even and odd parts",
                picard_sweeps_per_cell=sweeps / a.steps / ncells)

    # end to end through the C ABI: per step, H2D of the solution from pinned
    # host memory, one time step, D2H of the solution
    e2e = None
    if not a.no_e2e:
        nbytes = int(np.prod(m.solution_shape)) * 8
        pin_in = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
        pin_out = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
        pin_in.numpy()[:] = m.get_solution().reshape(-1)
        ke = max(1, a.steps)  # the same number of steps as the device-timed value
        # streamed: every step uploads its input and downloads its result, the
        # copies of neighbouring steps overlapping its compute
        m.step_io(pin_in.data_ptr(), 1, pin_out.data_ptr(), 1, nbytes, 2)  # warm-up (staging buffers)
        m.synchronize()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        m.step_io(pin_in.data_ptr(), 1, pin_out.data_ptr(), 1, nbytes, ke)
        f1.record(stream)
        f1.synchronize()
        e2e_ms = reduce_max(f0.elapsed_time(f1), world, dev)
        # the same one step at a time: upload, step, download, in order
        barrier()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(ke):
            m.upload_solution_async(pin_in.data_ptr(), nbytes)
            m.step(1)
            m.download_solution_async(pin_out.data_ptr(), nbytes)
        g1.record(stream)
        g1.synchronize()
        ser_ms = reduce_max(g0.elapsed_time(g1), world, dev)
        e2e = {"value": dof_per_step() * ke * world / (e2e_ms / 1e3), "unit": "DoF-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": ke,
               "api": "exa_mesh_step_io: per step H2D of the step's input from pinned memory, the step, D2H of its "
                      "result; the copies of steps k+1 and k-1 overlap step k",
               "serial": {"value": dof_per_step() * ke * world / (ser_ms / 1e3), "unit": "DoF-updates/s",
                          "api": "exa_mesh_copy_solution(H2D) + exa_mesh_step(1) + exa_mesh_copy_solution(D2H)"}}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        r = cpu_reference_run(3, 1, nthreads, runs=5)
        if r is not None:
            cpu = {"value": r["value"], "unit": "DoF-updates/s", "cores": nthreads, "kind": "reference",
                   "cpu": r["cpu"], "build": r["build"],
                   "sample": "median of 5 runs of 3 full time steps of the 27^3 mesh (after 1 warm-up step) on the "
                             "reference's generic kernels, %.1f s per run" % r["seconds"]}
    launches = sum(v[1] for v in ph.values())
    mixed = None if a.no_mixed else run_mixed_arm(a, u0, s.variant, dev)
    fused = None if a.no_fused else run_fused_arm(a, u0, s.variant, dev)
    lim = None if a.no_limiter else run_limiter_workload(a, world, dev, rank)
    ens = None if a.no_ensemble else run_ensemble_workload(a, world, dev, rank)
    ela = None if a.no_elastic else run_elastic_workload(a, world, dev, rank, fp64_peak)
    amr = None if a.no_amr else run_amr_workload(a, world, dev, rank)
    refined = None if a.no_refined else run_refined_workload(a, world, dev, rank)
    srv = None if a.no_serving else run_serving_workload(a, world, dev, rank)
    line = {
        "metric": METRIC, "value": value, "unit": "DoF-updates/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_total / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian pulses)",
        "config": {"workload": WORKLOAD, "dim": DIM, "order": ORDER, "cells": list(CELLS),
                   "dof_per_step": dof_per_step(), "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (solution 170 MB, face data 142 MB)"},
        "roofline": roof, "kernels": kernels, "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": int(launches),
        "clocks": clocks, "picard_sweeps_per_step": sweeps / a.steps, "predictor_variant": tune,
        "mixed": mixed, "fused": fused, "limiter": lim, "ensemble": ens, "serving": srv, "elastic": ela, "amr": amr, "refined": refined,
    }
    line["summary"] = summary(line)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _r(x, n=4):
    """x rounded to n significant digits (None stays None)"""
    if x is None:
        return None
    if isinstance(x, (bool, int)):
        return x
    return float("%.*g" % (n, x))


def summary(line):
    """The headline and every secondary workload's main figures in a few
    hundred characters: the last key of the line, so that a reader who only
    keeps the end of the line still sees them all."""
    g = lambda d, *ks: None if d is None else (d.get(ks[0]) if len(ks) == 1 else g(d.get(ks[0]), *ks[1:]))
    k = line.get("kernels", {})
    out = {"fp64_step": {"value": _r(line["value"]), "ms": _r(line["ms_per_step"]),
                         "frac": {n: _r(g(k, n, "frac"), 3) for n in ("predictor", "riemann", "corrector")}},
           "e2e": _r(g(line, "e2e", "value")), "cpu_ref": _r(g(line, "cpu_baseline", "value"))}
    if line.get("mixed"):
        m = line["mixed"]
        out["mixed"] = {"value": _r(m["value"]), "rel_l2_vs_fp64": _r(m["rel_l2_vs_fp64"], 2)}
    if line.get("fused"):
        out["fused"] = {"value": _r(line["fused"]["value"]), "reruns": line["fused"]["reruns_in_timed_steps"]}
    if line.get("limiter"):
        m = line["limiter"]
        out["limiter"] = {"value": _r(m["value"]), "steps": m["steps"], "irregular": m["irregular_steps"],
                          "ms": _r(m["ms_per_step"]), "cpu_ref": _r(g(m, "cpu_baseline", "value"))}
    if line.get("ensemble"):
        m = line["ensemble"]
        out["ensemble"] = {"value": _r(m["value"]), "one_at_a_time": _r(m["one_at_a_time"]["value"]),
                           "path": m.get("path")}
    if line.get("serving"):
        m = line["serving"]
        out["serving"] = {"p50_s": _r(m["p50_time_to_solution_s"], 3), "p99_s": _r(m["p99_time_to_solution_s"], 3),
                          "value": _r(m["value"]), "full_size": m.get("full_size"),
                          "one_at_a_time": {"p50_s": _r(m["one_at_a_time"]["p50_time_to_solution_s"], 3),
                                            "p99_s": _r(m["one_at_a_time"]["p99_time_to_solution_s"], 3),
                                            "value": _r(m["one_at_a_time"]["value"])}}
    if line.get("elastic"):
        m = line["elastic"]
        out["elastic"] = {"value": _r(m["value"]), "predictor_frac": _r(g(m, "kernels", "predictor", "frac"), 3),
                          "cpu_ref": _r(g(m, "cpu_baseline", "value"))}
    if line.get("refined"):
        out["refined"] = {"value": _r(line["refined"]["value"])}
    if line.get("amr"):
        out["amr_frac"] = {n: _r(g(line["amr"], n, "frac"), 3) for n in
                           ("volume_prolongation", "volume_restriction", "plot_vertices")}
    return out


def run_elastic_workload(a, world, dev, rank, fp64_peak=None):
    """The linear-kernel workload: 3D elastic waves (velocity pulse in a
    smoothly heterogeneous medium), N = 5 on 27^3 periodic cells; warm-up
    steps, then min(steps, 20) timed steps with CUDA events on the mesh
    stream, per-phase events for the kernel split; max over ranks."""
    import torch
    import exahype_b200 as eb
    from exahype_b200 import problems
    u0, _ = problems.elastic_pulse(EL_DIM, EL_ORDER, EL_CELLS, seed=SEED + rank)
    ncells = int(np.prod(EL_CELLS))
    s = eb.Solver(EL_DIM, EL_ORDER, eb.PDE_ELASTIC)
    chosen, vms = s.autotune(ncells)
    m = eb.Mesh(s, EL_CELLS, [0.0] * EL_DIM, [1.0] * EL_DIM, eb.BC_PERIODIC)
    m.set_solution(u0)
    m.init(0.0)
    stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
    m.step(max(3, a.warmup))
    m.synchronize()
    k = max(1, min(a.steps, 20))
    m.phase_times(reset=True)
    m.set_profiling(True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(k)
    e1.record(stream)
    e1.synchronize()
    m.set_profiling(False)
    ph = m.phase_times(reset=True)
    ms = reduce_max(e0.elapsed_time(e1), world, dev)
    dof_step = ncells * (EL_ORDER + 1) ** EL_DIM * EL_NVAR
    pred_ms = ph["predictor"][0] / k
    pfl = linear_predictor_flops(EL_DIM, EL_ORDER, ncells)
    ach = pfl / (pred_ms / 1e3) / 1e12
    peaks = load_peaks()
    byt = bytes_per_step(EL_DIM, EL_ORDER, ncells, nV=EL_NVAR, nD=EL_NDATA)
    # the linear Riemann solver reads both sides' states and writes both fluctuations
    F = (EL_ORDER + 1) ** (EL_DIM - 1)
    byt["riemann"] = 8 * ncells * EL_DIM * (2 * F * EL_NDATA + 2 * F * EL_NVAR)
    kern = {"predictor": dict(bound="fp64", achieved=ach, unit="TFLOP/s", ms=pred_ms, peak=fp64_peak,
                              frac=(ach / fp64_peak) if fp64_peak else None, algorithmic_flops_per_launch=pfl)}
    for name in ("riemann", "corrector"):
        t_ms = ph[name][0] / k
        gbs = byt[name] / (t_ms / 1e3) / 1e9
        kern[name] = dict(bound="hbm", achieved=gbs, unit="GB/s", ms=t_ms, peak=peaks["hbm_gbs"],
                          frac=gbs / peaks["hbm_gbs"])
    out = {"workload": EL_WORKLOAD, "value": dof_step * k * world / (ms / 1e3), "unit": "DoF-updates/s",
           "steps": k, "ms_per_step": ms / k, "dof_per_step": dof_step, "kernels": kern,
           "predictor_variant": {"chosen": chosen, "variant_ms_full_mesh": vms[:2]},
           "dt": m.state()["dt"], "timing": "exa_mesh_step(k), CUDA events on the mesh stream"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import pyoracle
        if pyoracle.ref_available(EL_DIM):
            nthreads = os.cpu_count() or 1
            r = pyoracle.Mesh(EL_DIM, EL_ORDER, EL_CELLS, [1.0] * EL_DIM, -1, pde=2, impl=ref_build()[0],
                             nthreads=nthreads)
            r.set_solution(u0)
            r.init(0.0)
            t0 = time.perf_counter()
            r.step(1)
            el = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": dof_step / el, "unit": "DoF-updates/s", "cores": nthreads,
                                   "kind": "reference", "build": ref_build()[1],
                                   "sample": "1 full time step of the 27^3 elastic mesh on the "
                                   "reference's linear kernels, %.1f s" % el}
    return out


def run_refined_workload(a, world, dev, rank):
    """A statically refined mesh (exa_mesh_create_refined): 3D Euler N=5, the
    27^3 periodic pulse mesh with its central 9^3 coarse cells refined once
    (18,954 coarse + 19,683 fine cells), global time steps; warm-up steps,
    then min(steps, 20) timed steps with CUDA events on the mesh stream and
    the per-phase split (the predictor phase includes the ancestors' face
    restriction and the descendants' face prolongation); max over ranks. CPU
    baseline: one step of a 9^3 mesh with its central 3^3 cells refined
    (1,431 cells) through the reference's kernels compiled from its sources,
    driven per cell by the oracle's refined-mesh sequencing on one thread."""
    import torch
    import exahype_b200 as eb
    from exahype_b200 import problems
    cells, lo, hi = (27, 27, 27), (9, 9, 9), (18, 18, 18)
    u0 = problems.pulse_refined(3, 5, cells, lo, hi, seed=SEED + rank)
    s = eb.Solver(3, 5, eb.PDE_EULER)
    if a.variant is not None:
        s.variant = a.variant
    else:
        s.autotune(4096)
    m = eb.Mesh.refined(s, cells, [0.0] * 3, [1.0] * 3, lo, hi)
    m.set_solution(u0)
    m.init(0.0)
    stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
    m.step(max(3, a.warmup))
    m.synchronize()
    st0 = m.state()
    k = max(1, min(a.steps, 20))
    m.phase_times(reset=True)
    m.set_profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(k)
    e1.record(stream)
    e1.synchronize()
    m.set_profiling(False)
    ph = m.phase_times(reset=True)
    ms = reduce_max(e0.elapsed_time(e1), world, dev)
    dof_step = m.ncells * 6 ** 3 * 5
    out = {"workload": "euler3d_N5_27^3_periodic_central_9^3_refined_once", "cells": m.ncells,
           "value": dof_step * k * world / (ms / 1e3), "unit": "DoF-updates/s", "steps": k, "ms_per_step": ms / k,
           "dof_per_step": dof_step, "predictor_variant": s.variant,
           "phase_ms_per_step": {n: v[0] / k for n, v in ph.items()},
           "picard_sweeps_per_step": (m.state()["picard_sweeps"] - st0["picard_sweeps"]) / k,
           "timing": "exa_mesh_step(k) on the refined mesh, CUDA events on the mesh stream"}
    # one regrid (exa_mesh_regrid): the refined box moved by 3 coarse cells
    # along x -- host topology, copies, prolongations, restrictions, the new
    # step size and the predictor of every cell; host wall clock
    m.synchronize()
    t0 = time.perf_counter()
    m.regrid([(0, (12, 9, 9), (21, 18, 18))])
    m.synchronize()
    out["regrid"] = {"ms": (time.perf_counter() - t0) * 1e3, "cells_after": m.ncells,
                     "what": "the central 9^3 refined box moved by 3 coarse cells along x (host wall clock, "
                             "topology build, data transfer, new step size and predictor included)"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import pyoracle
        if pyoracle.ref_available(3):
            sc, sl, sh = (9, 9, 9), (3, 3, 3), (6, 6, 6)
            r = pyoracle.RefinedMesh(3, 5, sc, [1.0] * 3, sl, sh, impl=ref_build()[0])
            r.set_solution(problems.pulse_refined(3, 5, sc, sl, sh, seed=SEED))
            r.init(0.0)
            t0 = time.perf_counter()
            r.step(1)
            el = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": r.ncells * 6 ** 3 * 5 / el, "unit": "DoF-updates/s", "cores": 1,
                                   "kind": "reference", "build": ref_build()[1],
                                   "sample": "1 step of a 9^3 mesh with its central 3^3 cells "
                                   "refined (%d cells), the reference's kernels per cell, %.1f s" % (r.ncells, el)}
    return out


def run_amr_workload(a, world, dev, rank):
    """AMR transfers and plotting on the 3D N=5 Euler shape: the 27^3 cells
    of a 9^3 coarse mesh refined once (levelDelta 1): prolongation of every
    fine cell from its parent, restriction of all of them back into the
    parents (atomic accumulation), the equidistant vertex projection of the
    fine mesh; CUDA events, median of 5 launches each after 2 warm-ups.
    Bytes per launch: the fine data written (read) once, the coarse data
    read (accumulated) once."""
    import torch
    import exahype_b200 as eb
    N, dim, nd = 5, 3, NVAR
    P = (N + 1) ** dim
    s = eb.Solver(dim, N, eb.PDE_EULER)
    nc, nf = 9 ** 3, 27 ** 3
    rng = np.random.default_rng(SEED)
    coarse = torch.as_tensor(rng.normal(size=(nc, P * nd))).to(dev)
    fine = torch.empty((nf, P * nd), dtype=torch.float64, device=dev)
    fid = np.arange(nf, dtype=np.int32)
    fx, fy, fz = fid % 27, (fid // 27) % 27, fid // 729
    par = ((fz // 3) * 81 + (fy // 3) * 9 + (fx // 3)).astype(np.int32)
    idx = np.stack([fx % 3, fy % 3, fz % 3], axis=1).astype(np.int32)
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x)).to(dev)
    fid_d, par_d, ld_d, idx_d = t(fid), t(par), t(np.ones(nf, dtype=np.int32)), t(idx)
    verts = torch.empty_like(fine)
    st = torch.cuda.current_stream(dev)

    def timed(fn):
        ms = []
        for r in range(7):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            e1.synchronize()
            if r >= 2:
                ms.append(e0.elapsed_time(e1))
        return reduce_max(float(np.median(ms)), world, dev)

    pro = timed(lambda: s.volume_unknowns_prolongation(fine, coarse, nf, fid_d, par_d, ld_d, idx_d))
    res = timed(lambda: s.volume_unknowns_restriction(coarse, fine, nf, fid_d, par_d, ld_d, idx_d))
    plo = timed(lambda: s.plot_vertices(fine, verts, nf))
    peaks = load_peaks()
    fb, cb = nf * P * nd * 8, nc * P * nd * 8

    def k(ms, by):
        gbs = by / (ms / 1e3) / 1e9
        return dict(ms=ms, bytes=by, achieved=gbs, unit="GB/s", peak=peaks["hbm_gbs"], frac=gbs / peaks["hbm_gbs"])

    return {"workload": "amr_euler3d_N5_9^3_to_27^3", "transfers": nf,
            "volume_prolongation": k(pro, fb + cb), "volume_restriction": k(res, fb + cb),
            "plot_vertices": k(plo, 2 * fb), "timing": "median of 5 launches, CUDA events"}


def run_limiter_workload(a, world, dev, rank):
    """The limiter workload to t = 0.2 (after init), timed with CUDA events on
    the mesh stream; max over ranks. DoF-updates/s counts every cell (DG or
    FV-limited) as (N+1)^2 nodes x 5 variables per step."""
    import torch
    import exahype_b200 as eb
    from exahype_b200 import problems
    luh, fv, _ = problems.explosion(LIM_DIM, LIM_ORDER, LIM_CELLS, seed=SEED + rank)
    s = eb.Solver(LIM_DIM, LIM_ORDER, eb.PDE_EULER)
    if a.variant is not None:
        s.variant = a.variant
    else:
        s.autotune(int(np.prod(LIM_CELLS)))
    m = eb.LimitingMesh(s, LIM_CELLS, [0.0] * LIM_DIM, [1.0] * LIM_DIM, eb.BC_OUTFLOW, helper_layers=1, cure_steps=0)
    m.set_solution(luh)
    m.set_fv_initial(fv)
    m.init(0.0)
    m.synchronize()
    stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if a.limiter_steps:
        m.step(a.limiter_steps)
        n = a.limiter_steps
    else:
        n = m.run_until(LIM_TEND)
    e1.record(stream)
    e1.synchronize()
    ms = reduce_max(e0.elapsed_time(e1), world, dev)
    st = m.state()
    status = m.status()
    dof_step = int(np.prod(LIM_CELLS)) * (LIM_ORDER + 1) ** LIM_DIM * NVAR
    out = {"workload": LIM_WORKLOAD, "value": dof_step * n * world / (ms / 1e3), "unit": "DoF-updates/s",
           "steps": n, "ms_per_step": ms / max(n, 1), "t_end": st["t"], "irregular_steps": st["irregular_steps"],
           "picard_sweeps": st["picard_sweeps"], "final_status_counts": np.bincount(status, minlength=4).tolist(),
           "predictor_variant": s.variant,
           "timing": "exa_lmesh_run_until(0.2): the step captured once as a CUDA graph (capture inside the "
                     "timed region), replayed 16 steps per host check of t, CUDA events"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import pyoracle
        if pyoracle.ref_available(LIM_DIM):
            nthreads = os.cpu_count() or 1
            r = pyoracle.RefLimitingMesh(LIM_DIM, LIM_ORDER, LIM_CELLS, [1.0] * LIM_DIM, 0, nthreads=nthreads,
                                         fast=ref_build()[0] == "ref_fast")
            r.set_solution(luh)
            r.set_fv_initial(fv)
            r.init(0.0)
            k = 8
            t0 = time.perf_counter()
            r.step(k)
            el = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": dof_step * k / el, "unit": "DoF-updates/s", "cores": nthreads,
                                   "kind": "reference", "build": ref_build()[1],
                                   "sample": "the first %d steps of the same workload on the reference's "
                                             "limiter/MUSCL-Hancock/ADER-DG kernels, %.1f s" % (k, el)}
    return out


def run_ensemble_workload(a, world, dev, rank, steps=50):
    """The ragged ensemble: 256 independent 2D periodic pulse solves (sides
    {9,27,81}, N {3,5,7}, per-instance seeded centre and amplitude
    U[0.1,0.5]), `steps` steps each, as one exa_batch (one CUDA graph launch
    per step) and, for comparison, one instance at a time on its own Mesh.
    Initialisation is outside both timed regions."""
    import torch
    import exahype_b200 as eb
    from exahype_b200 import problems
    ens = problems.pulse_ensemble(256, seed=SEED + rank)
    dofs = sum(int(np.prod(p["cells"])) * (p["order"] + 1) ** 2 * NVAR for p in ens)
    bt = eb.Batch()
    for p in ens:
        bt.add(2, p["order"], p["cells"], [1.0, 1.0], eb.BC_PERIODIC, p["luh"])
    bt.commit()
    bt.step(1)  # captures the graph
    bt.synchronize()
    stream = torch.cuda.ExternalStream(bt.stream_handle, device=dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bt.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms_b = reduce_max(e0.elapsed_time(e1), world, dev)
    # one at a time: the same problems, each on its own Mesh (same variants)
    solvers = {}
    ms_s = 0.0
    for p in ens:
        o = p["order"]
        if o not in solvers:
            solvers[o] = eb.Solver(2, o)
            solvers[o].variant = bt.variant(2, o)
        m = eb.Mesh(solvers[o], p["cells"], [0.0, 0.0], [1.0, 1.0], eb.BC_PERIODIC)
        m.set_solution(p["luh"])
        m.init(0.0)
        m.step(1)
        m.synchronize()
        st = torch.cuda.ExternalStream(m.stream_handle, device=dev)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(st)
        m.step(steps)
        f1.record(st)
        f1.synchronize()
        ms_s += f0.elapsed_time(f1)
        del m
    ms_s = reduce_max(ms_s, world, dev)
    counts = {}
    for p in ens:
        k = "N%d_%dx%d" % (p["order"], p["cells"][0], p["cells"][1])
        counts[k] = counts.get(k, 0) + 1
    return {"workload": "euler2d_pulse_ensemble_256_sides9-27-81_N3-5-7_periodic", "steps": steps,
            "instances": len(ens), "dof_per_step": dofs, "value": dofs * steps * world / (ms_b / 1e3),
            "unit": "DoF-updates/s", "ms_per_step": ms_b / steps,
            "one_at_a_time": {"value": dofs * steps * world / (ms_s / 1e3), "ms_per_step": ms_s / steps},
            "speedup_vs_one_at_a_time": ms_s / ms_b, "path": "fp64", "instance_mix": counts,
            "timing": "CUDA events on the batch stream (one graph launch per step) vs the sum over instances "
                      "of each Mesh's own stepping time"}


def run_serving_workload(a, world, dev, rank):
    """Continuous-batching serving of a seeded Poisson stream of independent
    Euler solves (exahype_b200.serving) against the same requests served one
    at a time on the plain FP64 path. Default mix (the full ranges): 32
    requests at 10/s, 70 % 2D with 27..243 cells per side, 30 % 3D with
    9..81, N in {3,5,7}, 20 % limiter explosions, 10..200 steps, 120 GB
    device budget; --serving-small uses 3D sides 9..27, 10..100 steps, 48
    requests at 40/s and a 64 GB budget. Initial data are built once, before
    any timing; a warm-up pass serves the same stream with one step per
    request (module loading, memory-pool growth to the mix's peak)."""
    from exahype_b200 import serving
    import exahype_b200 as eb
    small = a.serving_small
    kw = dict(sides_2d=(27, 243), sides_3d=(9, 27) if small else (9, 81), steps=(10, 100) if small else (10, 200))
    n, rate, budget = (48, 40.0, 64e9) if small else (32, 10.0, 120e9)
    variants = {}
    for dim in (2, 3):
        for o in (3, 5, 7):
            variants[(dim, o)] = eb.Solver(dim, o).autotune(4096)[0]
    reqs0 = serving.request_stream(n, rate, seed=SEED + rank, **kw)
    sizer = serving.Server(budget, variants)
    for r in reqs0:
        if sizer.bytes_for(r) <= budget:  # a request over the budget is rejected unbuilt
            r.build_initial()

    def clone(rs, steps=None):
        out = []
        for r in rs:
            c = serving.Request(r.rid, r.arrival, r.dim, r.order, r.cells, r.kind, steps or r.steps, r.seed)
            c.luh, c.fv = r.luh, r.fv
            out.append(c)
        return out

    serving.Server(budget, variants).run(clone(reqs0, steps=1), keep_results=False)
    reqs = clone(reqs0)
    srv = serving.Server(budget, variants)
    t0 = time.perf_counter()
    done, rejected = srv.run(reqs, keep_results=False)
    wall = time.perf_counter() - t0
    res = serving.summarise(done, wall)
    rej = {r.rid for r in rejected}
    base = clone([r for r in reqs0 if r.rid not in rej])
    t0 = time.perf_counter()
    serving.run_one_at_a_time(base, variants, keep_results=False)
    wall_b = time.perf_counter() - t0
    res_b = serving.summarise(base, wall_b)
    kinds = {}
    for r in reqs:
        k = "%dD_%s" % (r.dim, r.kind)
        kinds[k] = kinds.get(k, 0) + 1
    return {"workload": "serving_poisson_%d_requests" % n, "full_size": not small, "rate_per_s": rate,
            "budget_bytes": budget, "rejected_over_budget": len(rejected), "mix": kinds,
            "sides_3d": list(kw["sides_3d"]), "steps_range": list(kw["steps"]),
            "p50_time_to_solution_s": res["p50_s"], "p99_time_to_solution_s": res["p99_s"],
            "value": res["value"], "unit": "DoF-updates/s", "wall_s": wall,
            "one_at_a_time": {"p50_time_to_solution_s": res_b["p50_s"], "p99_time_to_solution_s": res_b["p99_s"],
                              "value": res_b["value"], "wall_s": wall_b},
            "timing": "host wall clock from the first arrival to the last result on the host, after a warm-up "
                      "pass of the same stream with one step per request (module loading, memory-pool growth)"}


def run_mixed_arm(a, u0, fp64_variant, dev):
    """The same workload with the mixed-precision predictor (EXA_PREDICTOR_MIXED):
    DoF-updates/s over the same timed steps, and the relative L2 difference of
    its solution from the FP64 path's after warm-up + timed steps."""
    import torch
    import exahype_b200 as eb
    out = {}
    sols = {}
    for name, variant in (("mixed", eb.PREDICTOR_MIXED), ("fp64", fp64_variant)):
        s = eb.Solver(DIM, ORDER, eb.PDE_EULER)
        s.variant = variant
        m = eb.Mesh(s, CELLS, [0.0] * DIM, [1.0] * DIM, eb.BC_PERIODIC)
        m.set_solution(u0)
        m.init(0.0)
        m.step(a.warmup)
        m.synchronize()
        stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.step(a.steps)
        e1.record(stream)
        e1.synchronize()
        sols[name] = m.get_solution()
        if name == "mixed":
            ms = e0.elapsed_time(e1)
            out = {"value": dof_per_step() * a.steps / (ms / 1e3), "unit": "DoF-updates/s",
                   "ms_per_step": ms / a.steps, "variant": variant,
                   "picard_sweeps_per_step": m.state()["picard_sweeps"] / (a.steps + a.warmup + 1)}
    err = float(np.linalg.norm(sols["mixed"] - sols["fp64"]) / np.linalg.norm(sols["fp64"]))
    out["rel_l2_vs_fp64"] = err
    out["within_1e-9"] = err <= 1e-9
    return out


def run_fused_arm(a, u0, variant, dev):
    """The same workload under fused time stepping (exa_mesh_init_fused,
    weight 0.99): the predictor runs right after the update with the
    estimated step, and a predictor rerun (a launch gated by a device count)
    follows the step bookkeeping. DoF-updates/s over the same number of timed
    steps, the reruns, and the update + predictor time per step."""
    import torch
    import exahype_b200 as eb
    s = eb.Solver(DIM, ORDER, eb.PDE_EULER)
    s.variant = variant
    m = eb.Mesh(s, CELLS, [0.0] * DIM, [1.0] * DIM, eb.BC_PERIODIC)
    m.set_solution(u0)
    m.init_fused(0.0, 0.99)
    m.step(a.warmup)
    m.synchronize()
    stream = torch.cuda.ExternalStream(m.stream_handle, device=dev)
    r0 = m.fused_state()["reruns"]
    m.phase_times(reset=True)
    m.set_profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(a.steps)
    e1.record(stream)
    e1.synchronize()
    m.set_profiling(False)
    ms = e0.elapsed_time(e1)
    ph = m.phase_times(reset=True)
    fs = m.fused_state()
    return {"value": dof_per_step() * a.steps / (ms / 1e3), "unit": "DoF-updates/s", "ms_per_step": ms / a.steps,
            "variant": variant, "weight": 0.99, "reruns_in_timed_steps": fs["reruns"] - r0,
            "update_plus_predictor_ms_per_step": (ph["corrector"][0] + ph["predictor"][0]) / a.steps,
            "timing": "exa_mesh_step under exa_mesh_init_fused, CUDA events on the mesh stream; the phase time is "
                      "the corrector and predictor launches, recorded with per-phase events in the same steps (the "
                      "predictor phase includes the gated rerun launch, whose blocks return at once unless the "
                      "estimate was too large)"}


def run_mixed_table(a, world, dev, rank):
    """The mixed-precision predictor (FP64 first sweep, FP32 increment sweeps;
    variants 4 and 5) against the FP64 path on each workload the mixed form
    is named for: per workload the FP64 (autotuned shape) and both mixed
    register budgets, CUDA events on the mesh stream, Picard sweeps per cell
    and step, and the mixed solution's relative L2 distance from the FP64
    one at the end. Workloads: the 27^3 N=5 3D pulses (20 steps), a 2D N=7
    81^2 pulse mesh (20 steps), the 81^2 N=5 explosion with the limiter
    (100 steps), and the 256-instance ragged 2D ensemble (20 steps). (3D N=7
    has no mixed form: its line-form working set does not fit in shared
    memory; the library rejects the variant there.)"""
    import torch
    import exahype_b200 as eb
    from exahype_b200 import problems

    def timed(m, k, stream_handle):
        st = torch.cuda.ExternalStream(stream_handle, device=dev)
        m.step(2)
        m.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        m.step(k)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    rows = []
    for name, dim, order, cells, steps, limiter in (
            ("euler3d_N5_27^3_pulses", 3, 5, (27, 27, 27), 20, False),
            ("euler2d_N7_81^2_pulse", 2, 7, (81, 81), 20, False),
            ("euler2d_N5_81^2_explosion_limiter", 2, 5, (81, 81), 100, True)):
        if limiter:
            u0, fv, _ = problems.explosion(dim, order, cells, seed=SEED)
        elif dim == 3:
            u0, _ = problems.gaussian_pulses_3d(order, cells, seed=SEED)
        else:
            u0, _ = problems.gaussian_pulse_2d(order, cells, seed=SEED)
        ncells = int(np.prod(cells))
        res, sols = {}, {}
        fp64_variant = eb.Solver(dim, order).autotune(min(4096, ncells))[0]
        for label, variant in (("fp64", fp64_variant), ("mixed", eb.PREDICTOR_MIXED),
                               ("mixed_2", eb.PREDICTOR_MIXED_2)):
            s = eb.Solver(dim, order)
            s.variant = variant
            if limiter:
                m = eb.LimitingMesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_OUTFLOW, helper_layers=1, cure_steps=0)
                m.set_solution(u0)
                m.set_fv_initial(fv)
            else:
                m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_PERIODIC)
                m.set_solution(u0)
            m.init(0.0)
            sw0 = m.state()["picard_sweeps"]
            ms = timed(m, steps, m.stream_handle)
            st = m.state()
            sols[label] = m.get_solution()
            res[label] = {"variant": variant, "ms_per_step": ms,
                          "sweeps_per_cell_step": (st["picard_sweeps"] - sw0) / ((steps + 2) * ncells)}
            del m
        for label in ("mixed", "mixed_2"):
            res[label]["rel_l2_vs_fp64"] = float(np.linalg.norm(sols[label] - sols["fp64"]) /
                                                 np.linalg.norm(sols["fp64"]))
            res[label]["speed_vs_fp64"] = res["fp64"]["ms_per_step"] / res[label]["ms_per_step"]
        rows.append(dict(workload=name, steps=steps, **res))
    # the ragged ensemble: every (dim, order) group with the mixed variant
    ens = problems.pulse_ensemble(256, seed=SEED + rank)
    out_e, sols = {}, {}
    for label in ("fp64", "mixed"):
        bt = eb.Batch()
        for p in ens:
            bt.add(2, p["order"], p["cells"], [1.0, 1.0], eb.BC_PERIODIC, p["luh"])
        bt.commit()
        if label == "mixed":
            for o in (3, 5, 7):
                bt.set_variant(2, o, eb.PREDICTOR_MIXED)
        bt.step(2)
        bt.synchronize()
        st = torch.cuda.ExternalStream(bt.stream_handle, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        bt.step(20)
        e1.record(st)
        e1.synchronize()
        out_e[label] = {"ms_per_step": e0.elapsed_time(e1) / 20, "sweeps": bt.sweeps()}
        sols[label] = [bt.get_solution(i) for i in range(len(ens))]
        del bt
    err = max(float(np.linalg.norm(a_ - b_) / np.linalg.norm(b_)) for a_, b_ in zip(sols["mixed"], sols["fp64"]))
    out_e["mixed"]["max_instance_rel_l2_vs_fp64"] = err
    out_e["mixed"]["speed_vs_fp64"] = out_e["fp64"]["ms_per_step"] / out_e["mixed"]["ms_per_step"]
    rows.append(dict(workload="euler2d_pulse_ensemble_256", steps=20, **out_e))
    return {"workload": "mixed_vs_fp64_table", "rows": rows,
            "timing": "CUDA events on the mesh / batch stream after 2 untimed steps"}


def measure_fp64_peak():
    """FP64 peaks measured in this run (TFLOP/s): the DFMA probe and the DMMA
    (mma.sync m8n8k4 f64) probe; the roofline uses the larger."""
    import ctypes
    import exahype_b200 as eb
    lib = eb.load()
    out = {}
    for name, fn in (("dfma", "exa_fp64_peak_probe"), ("dmma", "exa_fp64_mma_peak_probe")):
        v = ctypes.c_double()
        if hasattr(lib, fn) and getattr(lib, fn)(ctypes.byref(v)) == 0:
            out[name] = v.value
    return out or None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-probe", action="store_true")
    ap.add_argument("--variant", type=int, default=None, help="predictor variant (default: autotune)")
    ap.add_argument("--no-limiter", action="store_true", help="skip the limiter workload")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision arm")
    ap.add_argument("--no-fused", action="store_true", help="skip the fused-time-stepping arm")
    ap.add_argument("--limiter-steps", type=int, default=0, help="limiter workload: K steps instead of t = 0.2")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched ensemble workload")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving workload")
    ap.add_argument("--serving-small", action="store_true",
                    help="serving: the reduced request mix (3D sides 9..27, 10..100 steps)")
    ap.add_argument("--no-elastic", action="store_true", help="skip the linear-kernel (elastic waves) workload")
    ap.add_argument("--no-amr", action="store_true", help="skip the AMR transfer / plotting workload")
    ap.add_argument("--no-refined", action="store_true", help="skip the statically refined mesh workload")
    ap.add_argument("--workload", default="headline",
                    choices=["headline", "limiter", "ensemble", "serving", "elastic", "amr", "refined", "mixed-table"],
                    help="limiter / ensemble / serving / elastic / amr / refined: only that workload, as its own JSON line")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference_arm(a)
    if a.workload in ("limiter", "ensemble", "serving", "elastic", "amr", "refined", "mixed-table"):
        return run_secondary_only(a)
    return run_ours(a)


def run_secondary_only(a):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    run = {"limiter": run_limiter_workload, "ensemble": run_ensemble_workload,
           "serving": run_serving_workload, "elastic": run_elastic_workload, "amr": run_amr_workload,
           "refined": run_refined_workload, "mixed-table": run_mixed_table}[a.workload]
    if a.workload == "elastic":
        pk = None if a.no_fp64_probe else measure_fp64_peak()
        r = run(a, world, torch.device("cuda", local), rank, max(pk.values()) if pk else None)
    else:
        r = run(a, world, torch.device("cuda", local), rank)
    if rank == 0:
        print(json.dumps(dict(r, metric=METRIC, n_gpus=world, dtype="f64", data="synthetic (seeded)")), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
