#!/usr/bin/env python
"""Benchmark of the flat EZ field update on the 512^3 force-free turbulence
problem: cell-updates per second of the full LSRK(5,4) step (5 stages + the
Kreiss-Oliger pass) in FP32, with the algorithmic HBM bandwidth per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 512^3 interior points + 3 guards per side, periodic unit box,
dt = 0.5 dx, seeded random force-free turbulence (B = xhat + 32 Fourier modes
with |n| in [2, 8], |dB_k|^2 ~ k^-2, rms dB = 0.3; E = -v x B with an 8-mode
drift |v| <= 0.45), the semantics of the reference's CPU build.  The fields
(21 arrays x 556 MB resident) exceed the 126 MB L2 many times over, so no
L2 flush is needed between steps.

A "step" is one evolve_fields call over the whole grid.  The timed region is
K steps in one call of the library on the torch stream, bracketed by a
barrier and device synchronisation; with --gpus N (under torchrun) every rank
advances its own replica and the time is the max over ranks.

--impl reference times the reference's own CPU build (oracle/_ref, compiled
from its sources; else the oracle restatement) on the host cores: one
single-threaded process per core, each on a 512 x 512 x 8 periodic slab of
the same problem, aggregate cell-updates/s.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s & HBM GB/s per RK step; time-to-steady-state warm vs cold"
UNIT = "cell-updates/s"
N_SIDE = 512
# algorithmic bytes (FP32) per interior point: 112 per LSRK stage (read
# U[7] + dU[7], write U'[7] + dU'[7]); 56 for the KO pass; 616 per step
BYTES_STAGE = 112
BYTES_STEP = 616
SLAB_Z = 8
FP64_CHECK_STEPS = 1000  # the turbulence configuration's run length, for the FP32-vs-FP64 comparison


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profiled_traffic():
    """DRAM bytes per interior point of one stage launch, from the committed
    ncu summary (profiles/ez_stage_kernel.md), or None."""
    path = os.path.join(ROOT, "profiles", "ez_stage_kernel.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_point:\s*([0-9.]+)", txt)
    return float(m.group(1)) if m else None


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        time.sleep(0.4)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self, t0, t1):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sel = [ln for (ts, ln) in self.lines if t0 - 0.05 <= ts <= t1 + 0.15]
        if not sel:
            sel = [ln for (_, ln) in self.lines[-3:]]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in sel:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm.append(float(parts[2]))
                smax.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------- CPU reference

def _slab_input(tmpdir, steps_dtype="f32"):
    import numpy as np

    from coffee_b200 import problems
    from coffee_b200.fld import write_fld

    p = problems.turbulence_params(N_SIDE)
    p.N = [N_SIDE, N_SIDE, SLAB_Z]
    p.size = [1.0, 1.0, SLAB_Z / N_SIDE]
    f = problems.turbulence_fields(p, np.float32)
    path = os.path.join(tmpdir, "slab.fld")
    write_fld(path, f, guard=tuple(p.guard))
    cfg = os.path.join(tmpdir, "config.toml")
    p.write_toml(cfg)
    return p, path, cfg


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_run(steps: int, warmup: int, nproc: int | None = None):
    """Run the reference CPU build (or the restatement) on host cores.

    Returns dict(value, cores, kind, sample, seconds)."""
    from oracle import oracle

    cores = nproc or len(os.sched_getaffinity(0))
    cores = max(1, min(cores, 64))
    tmp = tempfile.mkdtemp(prefix="coffee_cpu_")
    try:
        p, fin, cfg = _slab_input(tmp)
        cells = N_SIDE * N_SIDE * SLAB_Z
        if oracle.reference_available():
            exe = oracle.ref_binary()
            env = dict(os.environ, COFFEE_ORACLE_CONFIG=cfg)
            procs = []
            for r in range(cores):
                out = os.path.join(tmp, f"out{r}.fld")
                procs.append(subprocess.Popen([exe, fin, out, str(steps), "--warmup", str(warmup)],
                                              cwd=tmp, env=env, stdout=subprocess.PIPE,
                                              stderr=subprocess.PIPE, text=True))
            secs = []
            for pr in procs:
                o, e = pr.communicate()
                if pr.returncode != 0:
                    raise RuntimeError(f"reference CPU build failed: {e[-500:]}")
                secs.append(json.loads(o.strip().splitlines()[-1])["seconds"])
            wall = max(secs)
            kind = "reference"
            sample = (f"{cores} concurrent single-threaded processes of the reference CPU build "
                      f"(oracle/_ref/coffee_ref_float), each a periodic {N_SIDE}x{N_SIDE}x{SLAB_Z} "
                      f"slab of the turbulence problem, {steps} timed steps after {warmup} warm-up")
        else:
            import numpy as np

            from coffee_b200.fld import read_fld

            f = [a.copy() for a in read_fld(fin).arrays]
            oracle.run_port(p, f, warmup)
            t0 = time.perf_counter()
            oracle.run_port(p, f, steps)
            wall = time.perf_counter() - t0
            cores = len(os.sched_getaffinity(0))
            kind = "port"
            sample = (f"oracle restatement (OpenMP, {cores} threads) on one periodic "
                      f"{N_SIDE}x{N_SIDE}x{SLAB_Z} slab, {steps} steps")
            cells = N_SIDE * N_SIDE * SLAB_Z
            return {"value": cells * steps / wall, "cores": cores, "kind": kind,
                    "sample": sample, "seconds": wall}
        return {"value": cells * cores * steps / wall, "cores": cores, "kind": kind,
                "sample": sample, "seconds": wall}
    finally:
        for fn in os.listdir(tmp):
            os.unlink(os.path.join(tmp, fn))
        os.rmdir(tmp)


# ------------------------------------------------------------------ arms

def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The largest value of x over all ranks (x itself with one rank)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells: int, steps: int, world: int, seconds_max: float) -> float:
    """Whole-job cell-updates/s: every rank advances its own replica of
    `cells` points by `steps` steps; the job takes the slowest rank's time."""
    return cells * steps * world / seconds_max


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference_arm(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    r = cpu_reference_run(args.steps, args.warmup)
    one = cpu_reference_run(args.steps, args.warmup, nproc=1)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * r["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random force-free turbulence)",
        "config": {"workload": "turbulence512 (CPU sample: 512x512x8 slabs)", "grid": [512, 512, 512],
                   "guard": 3, "periodic": True, "cfl": 0.5, "semantics": "reference CPU build",
                   "aggregate": ("P-core aggregate proxy: one single-threaded reference process "
                                 "per host core on its own periodic slab, no halo exchange")},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"], "cpu_model": cpu_model(),
                         "one_core": {"value": one["value"], "unit": UNIT, "cores": 1,
                                      "sample": one["sample"]}},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_gpu_arm(args):
    """The reference's own GPU build of field_solver_EZ (compiled from its
    sources into oracle/_ref/coffee_refgpu_float, single-rank device guard
    fill) on the same turbulence problem: a second, GPU-side baseline."""
    import numpy as np

    from coffee_b200 import problems
    from coffee_b200.solver import SimData, SimEnvironment
    from oracle import oracle

    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    p = problems.turbulence_params(args.n)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.init_fourier((1.0, 0.0, 0.0), *problems.turbulence_modes())
    f = data.download()
    data.close()
    env.close()
    # the reference's GPU build runs the GPU semantics (field_solver_EZ.cu)
    _, _, info = oracle.run_reference_gpu("ez", p, f, args.steps, warmup=args.warmup,
                                          timeout=3600)
    cells = args.n ** 3
    value = cells * args.steps / info["seconds"]
    line = {"impl": "reference-gpu", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * info["seconds"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random force-free turbulence, seed 20261203)",
            "config": {"workload": f"turbulence{args.n}", "grid": [args.n] * 3, "guard": 3,
                       "periodic": True, "cfl": 0.5,
                       "semantics": "reference GPU build (field_solver_EZ.cu)",
                       "build": ("oracle/_ref/coffee_refgpu_float: the reference's CUDA sources "
                                 "compiled for sm_100a, guard fill on the device")}}
    print(json.dumps(line), flush=True)
    return 0


class _DeviceArray:
    """A device array seen through __cuda_array_interface__ (zero-copy into torch)."""

    def __init__(self, ptr, shape, dtype):
        import numpy as np

        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def fp64_error(env, steps, modes, arith="reference"):
    """Per-field relative L2 (interior) between the FP32 and the FP64 run of
    the same algorithm from the same device initial condition after `steps`
    steps, in the benchmark's semantics (the reference CPU build's) and
    arithmetic.  The FP64 run uses the float build's 16 taper lanes: the
    CPU build offsets the taper's coordinates by its SIMD lane, and the lane
    count differs between its float (16) and double (8) builds."""
    import numpy as np
    import torch

    from coffee_b200.solver import FIELD_NAMES, FieldSolverEZ, SimData

    runs = {}
    for dtype in (np.float32, np.float64):
        d = SimData(env, dtype)
        d.init_fourier((1.0, 0.0, 0.0), *modes)
        sv = FieldSolverEZ(d, env, "cpu")
        sv.set_arithmetic(arith)
        sv.set_taper_lanes(16)
        # time advances as the drivers advance it: t += dt in the field precision
        t = dtype(0.0)
        dt = dtype(env.sim_params.dt)
        left = steps
        while left > 0:
            k = min(left, 100)
            sv.step(float(t), k)
            for _ in range(k):
                t = dtype(t + dt)
            left -= k
        sv.check_finite()
        runs[np.dtype(dtype).name] = (d, sv)
    g = list(env.grid().guard)
    d0, d1, d2 = env.dims
    out, rms, diff = {}, {}, {}
    for name in FIELD_NAMES:
        a = torch.as_tensor(_DeviceArray(runs["float32"][0].dev_ptr(name), (d2, d1, d0),
                                         np.float32), device="cuda")
        b = torch.as_tensor(_DeviceArray(runs["float64"][0].dev_ptr(name), (d2, d1, d0),
                                         np.float64), device="cuda")
        sl = (slice(g[2], d2 - g[2]), slice(g[1], d1 - g[1]), slice(g[0], d0 - g[0]))
        ai, bi = a[sl].double(), b[sl]
        den = torch.linalg.vector_norm(bi).item()
        dn = torch.linalg.vector_norm(ai - bi).item()
        out[name] = dn / den if den > 0 else 0.0
        rms[name] = den / math.sqrt(bi.numel())
        diff[name] = dn / math.sqrt(bi.numel())
        del a, b, ai, bi
    for d, sv in runs.values():
        sv.close()
        d.close()
    torch.cuda.synchronize()
    return out, rms, diff


def run_ours(args):
    import numpy as np
    import torch

    from coffee_b200 import problems
    from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment

    ws, rank, local = _dist()
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize(dev)

    n_side = args.n
    p = problems.turbulence_params(n_side)
    cells = n_side ** 3
    env = SimEnvironment(p, device=local)
    data = SimData(env, np.float32)
    modes = problems.turbulence_modes()
    data.init_fourier((1.0, 0.0, 0.0), *modes)
    solver = FieldSolverEZ(data, env, "cpu", stream=stream.cuda_stream)
    solver.set_arithmetic(args.arith)
    dt = np.float32(p.dt)

    # warm-up (untimed)
    t = np.float32(0.0)
    solver.step(float(t), args.warmup)
    for _ in range(args.warmup):
        t = np.float32(t + dt)
    barrier()

    clocks = ClockSampler(local)
    clocks.start()
    solver.set_timing(True)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    solver.step(float(t), args.steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    w1 = time.time()
    barrier()
    clk = clocks.stop(w0, w1)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, dist, dev)
    timing = solver.last_timing()
    solver.set_timing(False)
    solver.check_finite()

    # the other arithmetic of the same solver, timed the same way on rank 0
    # (its cost or gain beside the mode measured)
    other = None
    if ws == 1 and not args.no_arith_compare:
        alt = "fast" if args.arith == "reference" else "reference"
        solver.set_arithmetic(alt)
        solver.step(float(t), 1)
        torch.cuda.synchronize(dev)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        solver.step(float(t), args.steps)
        a1.record(stream)
        torch.cuda.synchronize(dev)
        other = {"mode": alt, "ms_per_step": a0.elapsed_time(a1) / args.steps}
        solver.set_arithmetic(args.arith)
        # the fields moved on: start the end-to-end leg from the device set-up
        data.init_fourier((1.0, 0.0, 0.0), *modes)

    value = job_throughput(cells, args.steps, ws, ms_max / 1e3)
    step_ms = ms_max / args.steps
    hbm_gbs = BYTES_STEP * cells / (step_ms / 1e3) / 1e9
    n_stage = timing["launches"]["stage"]
    avg_stage_ms = timing["ms"]["stage"] / max(1, n_stage)
    achieved = BYTES_STAGE * cells / (avg_stage_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()
    traffic_pp = _profiled_traffic()

    # ---- end to end through the public API with host buffers
    nbytes = 7 * data.env.dims[0] * data.env.dims[1] * data.env.dims[2] * 4
    host = torch.empty(nbytes // 4, dtype=torch.float32, pin_memory=True)
    hnp = host.numpy()
    data.download_packed(hnp)
    barrier()
    tt = np.float32(0.0)
    w0 = time.perf_counter()
    data.upload_packed(hnp)
    energies = []
    for _ in range(args.steps):
        solver.step(float(tt), 1)
        tt = np.float32(tt + dt)
        energies.append(solver.total_energy("B"))
    data.download_packed(hnp)
    torch.cuda.synchronize(dev)
    e2e_s = max_over_ranks(time.perf_counter() - w0, dist, dev)
    barrier()
    e2e_value = job_throughput(cells, args.steps, ws, e2e_s)
    d2h_diag = 8 * (148 * 4)  # FP64 partials read back per energy diagnostic

    err64 = None
    if rank == 0 and ws == 1 and not args.no_fp64_check:
        nck = args.fp64_steps
        rel, rms, diff = fp64_error(env, nck, modes, args.arith)
        err64 = {"steps": nck, "grid": [n_side] * 3,
                 "semantics": "reference CPU build, 16 taper lanes in both precisions",
                 "arithmetic": args.arith, "rel_l2": rel, "rms_fp64": rms, "rms_diff": diff,
                 "note": ("FP32 against FP64 of the same algorithm from the same FP64 initial "
                          "condition over the interior: relative L2, the FP64 field's rms and "
                          "the rms of the difference.  P, the divergence-cleaning potential, "
                          "stays at the truncation level of div B in FP64 (rms ~1e-10) and at "
                          "the level of FP32 rounding in FP32, so its relative error is large "
                          "while its absolute error is ~3e-8 against |B| ~ 1")}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        agg = cpu_reference_run(steps=2, warmup=1)
        one = cpu_reference_run(steps=2, warmup=1, nproc=1)
        cpu = {"value": agg["value"], "unit": UNIT, "cores": agg["cores"], "kind": agg["kind"],
               "sample": agg["sample"] + " (P-core aggregate proxy: no halo exchange)",
               "cpu_model": cpu_model(),
               "one_core": {"value": one["value"], "unit": UNIT, "cores": 1, "kind": one["kind"],
                            "sample": one["sample"]}}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random force-free turbulence, seed 20261203)",
            "config": {"workload": f"turbulence{n_side}", "grid": [n_side] * 3, "guard": 3,
                       "periodic": True, "cfl": 0.5, "semantics": "reference CPU build",
                       "l2": ("inputs larger than L2 (21 arrays x 556 MB resident), no flush"
                              if n_side >= 512 else "smaller case (profiling)"),
                       "parallelism": f"replicas x{ws}"},
            "hbm_gbs": hbm_gbs,
            "roofline": {"kernel": "ez_stage_kernel (LSRK stages 2-5)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (traffic_pp * cells if traffic_pp else None),
                         "algorithmic_bytes_per_launch": BYTES_STAGE * cells,
                         "avg_launch_ms": avg_stage_ms},
            "kernels_ms": {k: v for k, v in timing["ms"].items()},
            "kernel_launches": timing["launches"],
            "gpu_launches": sum(timing["launches"].values()),
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": nbytes / args.steps,
                    "d2h_bytes_per_step": nbytes / args.steps + d2h_diag},
            "arithmetic": {"mode": args.arith,
                           "note": ("reference: the float build's own operations and rounding, "
                                    "bit for bit; fast: regrouped, equal to rounding"),
                           "other": other},
            "cpu_baseline": cpu,
            "error_vs_fp64": err64,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    data.close()
    env.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------- other solvers' workloads
# Not the headline: measurement lines for the configurations of the other
# solvers (--workload gr-wald | logsph-batch | logsph | cyl-pulsar | yee-wave |
# yee-pulsar).  Their reference implementation exists only as the reference's
# GPU build, which --impl reference times on the same case.

# Algorithmic bytes per cell of the timed kernel: the LSRK stage kernels of
# the EZ solvers (GR: read D, B, P, dU, E and H, write D', B', P', dU' and
# the E', H' of the output, 20 + 20 arrays of 4 bytes; the sqrt(gamma)
# table, 4 more, is not counted); for the staggered solver the update pass
# of substeps 2-3,
# which reads E, B and their start-of-step copies and writes E*, B'
# (12 + 6 arrays of 4 bytes).
# The Kerr-Schild staggered solver's update pass reads E, H, B, the lowered
# B, rho, D and the start-of-step copies and writes D*, B' (22 + 6 arrays).
VARIANT_STAGE_BYTES = {"gr-wald": 160, "logsph-batch": 112, "logsph": 112, "cyl-pulsar": 112,
                       "yee-wave": 72, "yee-pulsar": 72, "gryee-wald": 112}


def _variant_cases(workload, n=512, batch_runs=64):
    """(list of (solver class name, params, FP32 fields), description); n is
    the grid side of the staggered workloads (512 is the benchmark),
    batch_runs the number of runs of the log-spherical batch (64 is the
    benchmark; the first runs of the seeded draw)."""
    import numpy as np

    from coffee_b200 import problems

    if workload == "gr-wald":
        p = problems.wald_params(N=256, half_size=20.0, a=0.9, pml=16)
        return [("FieldSolverGrEZ", "gr", p, problems.wald_fields(p, np.float32))], {
            "workload": "gr-wald256", "grid": [256] * 3, "spin": 0.9, "domain": [-20, 20],
            "pml": 16, "note": "Wald field B0 = 1 along the spin axis, E = 0, P = 0"}
    if workload == "yee-wave":
        p = problems.alfven_params(N=n, guard=2)
        p.dt = 0.3 / n
        return [("FieldSolver", "yee", p,
                 problems.alfven_plane_wave_fields(p, np.float32, yee=True))], {
            "workload": f"yee-alfven{n}", "grid": [n] * 3, "guard": 2,
            "solver": "staggered SSP-RK3 (field_solver)", "cfl": 0.3,
            "note": "plane Alfven wave on B0 = x-hat, k = 2 pi (2, 0, 1), periodic box"}
    if workload == "yee-pulsar":
        p = problems.pulsar_params(N=n, guard=2, half_size=64.0, radius=4.0, omega=0.05,
                                   pml=n // 16)
        p.dt = 0.3 * (128.0 / n)
        return [("FieldSolver", "yee", p, problems.pulsar_fields(p, np.float32, yee=True))], {
            "workload": f"yee-pulsar{n}", "grid": [n] * 3, "guard": 2,
            "solver": "staggered SSP-RK3 (field_solver)", "domain": [-64, 64], "radius": 4.0,
            "omega": 0.05, "pml": n // 16, "note": "rotating dipole star, absorbing layer"}
    if workload == "gryee-wald":
        p = problems.wald_params(N=256, half_size=20.0, a=0.9, pml=16)
        return [("FieldSolverGr", "gryee", p, problems.wald_fields(p, np.float32, yee=True))], {
            "workload": "gryee-wald256", "grid": [256] * 3, "spin": 0.9, "domain": [-20, 20],
            "pml": 16, "solver": "staggered SSP-RK3 in Kerr-Schild coordinates (field_solver_gr)",
            "note": "Wald field B = curl(x dy - y dx)/2 / sqrt(gamma), D = 0 (user_wald.hpp)"}
    if workload == "logsph":
        p = problems.sph_pulsar_params(nr=2048, nth=1024, guard=4, omega=0.2)
        return [("FieldSolverEZSpherical", "sph", p, problems.sph_pulsar_fields(p, np.float32))], {
            "workload": "logsph2048x1024", "grid": [2048, 1024], "r": [1, 100]}
    if workload == "cyl-pulsar":
        p = problems.cyl_pulsar_params(nR=1024, nz=2048, guard=3, R_max=64.0, radius=4.0)
        return [("FieldSolverEZCylindrical", "cyl", p, problems.cyl_pulsar_fields(p, np.float32))], {
            "workload": "cyl-pulsar1024x2048", "grid": [1024, 2048]}
    rng = np.random.default_rng(20261203)
    sizes = [(512, 256), (768, 384), (1024, 512), (2048, 1024)]
    runs = []
    for _ in range(batch_runs):
        nr, nth = sizes[int(rng.integers(len(sizes)))]
        r_lc = float(rng.uniform(3.0, 10.0))
        p = problems.sph_pulsar_params(nr=nr, nth=nth, guard=4, omega=1.0 / r_lc)
        runs.append(("FieldSolverEZSpherical", "sph", p, problems.sph_pulsar_fields(p, np.float32)))
    return runs, {"workload": f"logsph-batch{batch_runs}", "runs": batch_runs,
                  "grids": "r x theta drawn from 512x256, 768x384, 1024x512, 2048x1024 (seeded)",
                  "r": [1, 100], "R_LC": [3, 10], "launch": "one kernel per phase for all runs"}


def run_variant(args):
    import numpy as np
    import torch

    from coffee_b200 import solver as sv

    ws, rank, local = _dist()
    if args.impl == "reference":
        from oracle import oracle

        if rank != 0:
            return 0
        runs, cfg = _variant_cases(args.workload, args.n, args.batch_runs)
        secs, cells = 0.0, 0
        for _cls, name, p, f in runs:
            oracle.run_reference_gpu(name, p, f, args.warmup)
            _, _, info = oracle.run_reference_gpu(name, p, f, args.steps)
            secs += info["seconds"]
            cells += int(np.prod(p.N))
        value = cells * args.steps / secs
        line = {"impl": "reference", "metric": "cell-updates/s", "value": value, "unit": UNIT,
                "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": cfg,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": 0,
                                 "kind": "reference",
                                 "sample": "the reference's own GPU build of this solver "
                                           "(oracle/_ref/coffee_refgpu_float), one run at a "
                                           "time; the reference has no CPU build of it"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    runs, cfg = _variant_cases(args.workload, args.n, args.batch_runs)
    objs = []
    cells = 0
    for cls_name, _name, p, f in runs:
        env = sv.SimEnvironment(p, device=local)
        data = sv.SimData(env, np.float32)
        data.upload(f)
        solver = getattr(sv, cls_name)(data, env, stream=stream.cuda_stream)
        objs.append((env, data, solver))
        cells += int(np.prod(p.N))
    batch = sv.SphBatch([o[2] for o in objs], stream=stream.cuda_stream) \
        if args.workload == "logsph-batch" else None

    def advance(n):
        if batch is not None:
            batch.step(n)
        else:
            objs[0][2].step(0.0, n)

    advance(args.warmup)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    if batch is None:
        objs[0][2].set_timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop(w0, time.time())
    ms = e0.elapsed_time(e1)
    step_ms = ms / args.steps
    value = job_throughput(cells, args.steps, 1, ms / 1e3)
    peak, peak_kind = _peaks()
    if batch is None:
        timing = objs[0][2].last_timing()
        objs[0][2].set_timing(False)
        n_stage = timing["launches"]["stage"]
        avg = timing["ms"]["stage"] / max(1, n_stage)
        kname = {"gr-wald": "gr_stage_kernel (LSRK stages 2-5)",
                 "cyl-pulsar": "cyl_stage_kernel (LSRK stages 2-5)",
                 "logsph": "sph_stage_kernel (LSRK stages 2-5)",
                 "yee-wave": "yee_update_kernel (substeps 2-3)",
                 "yee-pulsar": "yee_update_kernel (substeps 2-3)",
                 "gryee-wald": "gyee_update_kernel (substeps 2-3)"}[args.workload]
        roof = {"kernel": kname, "bound": "hbm",
                "achieved": VARIANT_STAGE_BYTES[args.workload] * cells / (avg / 1e3) / 1e9,
                "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": VARIANT_STAGE_BYTES[args.workload] * cells,
                "avg_launch_ms": avg}
        launches = sum(timing["launches"].values())
        launch_note = "stage + KO kernels counted by the solver's launch hooks"
        if args.workload == "gr-wald":
            launches += 2  # the E, H passes of the call, over both field buffers
            launch_note += ", plus the two E, H passes of the call"
        if args.workload == "gryee-wald":
            launches = objs[0][2].launches_per_step() * args.steps
            launch_note = ("per substep: E/H, rho, shell, update and clamp passes, and the "
                           "E_par cleaning in the last")
        if args.workload.startswith("yee"):
            per_call = 0 if runs[0][2].problem == 1 else 1
            launches = objs[0][2].launches_per_step() * args.steps + per_call
            launch_note = ("per substep: shell copy, update and clamp passes; the star problem "
                           "adds three star passes and a guard pass (box problem: one guard pass "
                           "per call)")
    else:
        roof = {"kernel": "whole batched step (stage, axis and KO launches)", "bound": "hbm",
                "achieved": BYTES_STEP * cells / (step_ms / 1e3) / 1e9, "peak": peak,
                "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_step": BYTES_STEP * cells}
        launches = 13 * args.steps + 1
        launch_note = ("5 stage + 5 axis + 1 KO + 1 axis + 1 time-advance per step (one captured "
                       "CUDA graph, replayed per step), 1 axis per call")
        cfg["autotuned"] = batch.info()
    roof["frac"] = roof["achieved"] / peak
    # end to end: upload from pinned host memory, K steps, download
    hosts = []
    nbytes = 0
    for env, data, _s in objs:
        d0, d1, d2 = env.dims
        h = torch.empty(7 * d0 * d1 * d2, dtype=torch.float32, pin_memory=True)
        data.download_packed(h.numpy())
        hosts.append(h)
        nbytes += h.numel() * 4
    torch.cuda.synchronize(dev)
    w0 = time.perf_counter()
    for (env, data, _s), h in zip(objs, hosts):
        data.upload_packed(h.numpy())
    advance(args.steps)
    for (env, data, _s), h in zip(objs, hosts):
        data.download_packed(h.numpy())
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - w0
    line = {"metric": "cell-updates/s", "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg, "roofline": roof, "gpu_launches": launches,
            "gpu_launches_note": launch_note,
            "e2e": {"value": job_throughput(cells, args.steps, 1, e2e_s), "unit": UNIT,
                    "h2d_bytes_per_step": nbytes / args.steps,
                    "d2h_bytes_per_step": nbytes / args.steps},
            "clocks": clk}
    if batch is not None:
        # the persistent mode: every call one cooperative launch with bounded
        # grid-wide barriers between the phases (it synchronises per call)
        batch.set_persistent(True)
        advance(args.warmup)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        advance(args.steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        pms = e0.elapsed_time(e1)
        batch.set_persistent(False)
        line["persistent"] = {
            "ms_per_step": pms / args.steps,
            "value": job_throughput(cells, args.steps, 1, pms / 1e3),
            "frac": BYTES_STEP * cells / (pms / args.steps / 1e3) / 1e9 / peak,
            "launches": 2, "note": "per call: 1 axis launch, 1 cooperative launch of all steps"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if batch is not None:
        batch.close()
    for env, data, s in objs:
        s.close()
        data.close()
        env.close()
    return 0


# ------------------------------------------------------ learned warm start
# --workload surrogate: training steps of the 3D U-Net (coffee_b200/surrogate.py)
# on the library's BF16 tensor-core kernels: 8 samples of 64^3, forward +
# masked MSE + backward + Adam per step.  The roofline line is the largest
# convolution's forward kernel (48 -> 16 channels) against the measured
# dense BF16 tensor peak; --study adds the warm-start study.

def run_surrogate(args):
    import numpy as np
    import torch

    from coffee_b200 import surrogate as sg

    ws, rank, local = _dist()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the learned warm start has no "
                              "counterpart in the reference"}), flush=True)
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, side = 8, 64
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.standard_normal((n, side, side, side, sg.CIN)).astype(np.float32))
    x = x.to(dev).to(torch.bfloat16)
    tgt = torch.from_numpy(rng.standard_normal((n, side, side, side, sg.COUT)).astype(np.float32))
    tgt = tgt.to(dev)
    mask = torch.ones((n, side, side, side), device=dev)
    net = sg.UNet(seed=0, device=str(dev))

    def train_step():
        out = net.forward(x)
        _, dout = net.loss(out, tgt, mask)
        net.backward(dout)
        net.step(1e-3)

    for _ in range(args.warmup):
        train_step()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    w0 = time.time()
    e0.record(stream)
    for _ in range(args.steps):
        train_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop(w0, time.time())
    ms = e0.elapsed_time(e1) / args.steps
    vox = n * side ** 3
    def conv_time(fn, L, xin):
        z = torch.empty(xin.shape[:4] + (L.cout,), dtype=torch.float32, device=dev)
        a = torch.empty(xin.shape[:4] + (L.cout,), dtype=torch.bfloat16, device=dev)
        for _ in range(3):
            fn(xin, L.wb, L.b, L.cout, True, z, a)
        e0.record(stream)
        for _ in range(10):
            fn(xin, L.wb, L.b, L.cout, True, z, a)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / 10, 2.0 * 27 * L.cin * L.cout * xin[..., 0].numel()

    # the tcgen05 convolution of layer 4 (32 -> 32 channels, 32^3 x 8), and
    # the largest one, layer 5 (48 -> 16 channels at full size, mma.sync)
    conv_ms, flops = conv_time(sg.conv_forward_tc, net.layers[3], net._saved["a3"])
    mma_ms, mma_flops = conv_time(sg.conv_forward, net.layers[4], net._saved["cat"])
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        peak, kind = 1590.0, "fallback"
    achieved = flops / (conv_ms / 1e3) / 1e12

    # the weight gradient of the same two layers, tcgen05 against mma.sync
    def wgrad_time(fn, L, xin):
        dyb = torch.zeros(xin.shape[:4] + (L.cout,), dtype=torch.bfloat16, device=dev)
        dyb.normal_()
        wsb = torch.empty(sg.workspace_bytes(L.cout, L.cin), dtype=torch.uint8, device=dev)
        dw = torch.empty((L.cout, 27, L.cin), dtype=torch.float32, device=dev)
        for _ in range(3):
            fn(dyb, xin, dw, wsb)
        e0.record(stream)
        for _ in range(10):
            fn(dyb, xin, dw, wsb)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        t = e0.elapsed_time(e1) / 10
        return {"ms": t, "tflops": 2.0 * 27 * L.cin * L.cout * xin[..., 0].numel() / (t / 1e3) / 1e12}

    wgrad = {}
    for name, L, xin in (("32_32", net.layers[3], net._saved["a3"]),
                         ("48_16", net.layers[4], net._saved["cat"])):
        wgrad[name] = {"tcgen05": wgrad_time(sg.conv_backward_weight_tc, L, xin),
                       "mma_sync": wgrad_time(sg.conv_backward_weight, L, xin)}
    sg.check_tc()
    line = {"metric": "training voxels/s", "value": vox / (ms / 1e3), "unit": "voxels/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (random inputs and targets)",
            "config": {"workload": "surrogate-unet64", "samples": n, "grid": [side] * 3,
                       "channels": [sg.CIN, sg.C1, sg.C2, sg.COUT],
                       "step": "forward + masked MSE + backward + Adam, all on the library's kernels"},
            "roofline": {"kernel": "conv3d_fwd_tc_kernel (tcgen05 + TMA, 32 -> 32 channels, "
                                   "32^3 x 8)",
                         "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "peak_kind": kind, "frac": achieved / peak, "traffic": None,
                         "avg_launch_ms": conv_ms, "flops_per_launch": flops},
            "conv_48_16_mma_sync": {"ms": mma_ms, "tflops": mma_flops / (mma_ms / 1e3) / 1e12},
            "weight_gradient": wgrad,
            "gpu_launches": None, "clocks": clk}
    if args.study:
        # the configured oblique rotator: 384^3, R* = 12 and R_LC = 60 cells,
        # the network on the 128^3 grid of the same box (surrogate.rotator_study)
        line["warm_start_study"] = sg.rotator_study(n_train=args.study_train,
                                                    iters=args.study_iters)
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours",
                    help="reference-gpu: the reference's own GPU build on the turbulence problem")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=FP64_CHECK_STEPS,
                    help="length of the FP32-vs-FP64 comparison (rank 0, one GPU)")
    ap.add_argument("--arith", choices=["reference", "fast"], default="reference",
                    help="arithmetic of the flat solver (reference: the float build's own)")
    ap.add_argument("--no-arith-compare", action="store_true",
                    help="skip timing the other arithmetic beside the measured one")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the FP32-vs-FP64 error report of the turbulence run")
    ap.add_argument("--n", type=int, default=N_SIDE,
                    help="grid side of the turbulence and staggered workloads (512 is the "
                         "benchmark)")
    ap.add_argument("--workload", default="turbulence",
                    choices=["turbulence", "gr-wald", "logsph-batch", "logsph", "cyl-pulsar",
                             "yee-wave", "yee-pulsar", "gryee-wald", "surrogate"])
    ap.add_argument("--batch-runs", type=int, default=64,
                    help="runs of the logsph-batch workload (64 is the benchmark)")
    ap.add_argument("--study", action="store_true",
                    help="with --workload surrogate: also run the warm-start study")
    ap.add_argument("--study-train", type=int, default=40,
                    help="training runs (384^3 each) of the warm-start study")
    ap.add_argument("--study-iters", type=int, default=2000,
                    help="training iterations of the warm-start study")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.workload == "surrogate":
        return run_surrogate(args)
    if args.workload != "turbulence":
        return run_variant(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.impl == "reference-gpu":
        return run_reference_gpu_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
