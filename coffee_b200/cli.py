"""Command-line drivers: the reference's executables over this library.

    python -m coffee_b200 <driver> -c config.toml [-o DIR] [--restart FILE]
                          [--steps N] [--device D] [--precision f32|f64]

Each driver mirrors one of the reference's ``main-*.cpp`` programs: it reads
the same ``config.toml`` (``Coffee::sim_environment``, ``parse_config``,
``src/sim_params.cpp:7-146``), checks the problem id the program requires,
sets the initial condition of its ``user_*.hpp`` snippet, and runs the
reference's main loop (``src/main-alfven3d.cpp:56-125``): for step = 0 ..
max_steps, a snapshot every ``snapshot_interval`` steps, an output every
``data_interval`` steps, then ``evolve_fields(time)`` and time += dt.

| driver | reference program | problem | initial condition | solver |
|---|---|---|---|---|
| wave | main-wave.cpp | 0 | user_alfven.hpp | field_solver_EZ |
| emwave | (user_emwave.hpp) | 0 | user_emwave.hpp | field_solver_EZ |
| pulsar3d | main-pulsar3d.cpp | 1 | user_pulsar3d_EZ.hpp | field_solver_EZ |
| alfven3d | main-alfven3d.cpp | 2 | user_pulsar3d_EZ.hpp | field_solver_EZ |
| gr | main-gr.cpp | any | user_wald2.hpp | field_solver_gr_EZ |
| pulsar2d-spherical | main-pulsar2d-spherical.cpp | any | user_pulsar_sph.hpp | field_solver_EZ_spherical |
| pulsar2d-cylindrical | main-pulsar2d-cylindrical.cpp | any | user_pulsar.hpp | field_solver_EZ_cylindrical |
| wave-yee | main-wave.cpp without EZ | 0 | user_alfven.hpp (staggered branch) | field_solver |
| pulsar3d-yee | main-pulsar3d.cpp without EZ | 1 | user_pulsar3d.hpp | field_solver |
| alfven3d-yee | main-alfven3d.cpp without EZ | 2 | user_pulsar3d.hpp | field_solver |
| gr-yee | main-gr-Yee.cpp | any | user_wald.hpp | field_solver_gr |

Outputs go to DIR (default ``Data``): ``fld.NNNNN.fld`` holds E, B, P and
J, div E, div B of the output step on every ``downsample``-th interior point
(the reference's HDF5 ``fld.NNNNN.h5`` datasets, written in this library's
field-file format since HDF5 is not part of it); ``snapshot.NNNNN.fld`` is a
full restart state (``coffee_solver_save_snapshot``); ``energy.txt`` gets
one line ``step time Wb We`` per output (the energy file of
``main-wave.cpp``), Cartesian solvers only (the staggered solver's energies
interpolate every component to the vertices, as its total_energy does).  Steps between two events run as one
``coffee_solver_step`` call, which advances time exactly as the loop does.
With ``--energy-diag`` (flat drivers) the field files also hold the CPU
build's energy-change diagnostics dU_EgtB, dU_Epar, dU_KO, dU_EgtB_cum,
dU_Epar_cum, dU_KO_cum after J, div E, div B, and the _cum arrays are reset
to zero after each output, as the reference's exporter does
(``src/utils/data_exporter.cpp:624-638``).
"""
from __future__ import annotations

import argparse
import os
import sys
from dataclasses import dataclass

import numpy as np

from . import problems
from .config import SimParams
from .fld import write_fld

FLAT, GR, SPH, CYL, YEE, GRYEE = "flat", "gr", "sph", "cyl", "yee", "gryee"


@dataclass(frozen=True)
class Driver:
    name: str
    program: str
    problem: int | None  # required problem id (None: any)
    kind: str            # solver
    init: str            # problems.<init>(params, dtype)


DRIVERS = {d.name: d for d in (
    Driver("wave", "main-wave.cpp", 0, FLAT, "alfven_plane_wave_fields"),
    Driver("emwave", "user_emwave.hpp", 0, FLAT, "emwave_fields"),
    Driver("pulsar3d", "main-pulsar3d.cpp", 1, FLAT, "pulsar_fields"),
    Driver("alfven3d", "main-alfven3d.cpp", 2, FLAT, "pulsar_fields"),
    Driver("gr", "main-gr.cpp", None, GR, "wald_fields"),
    Driver("pulsar2d-spherical", "main-pulsar2d-spherical.cpp", None, SPH, "sph_pulsar_fields"),
    Driver("pulsar2d-cylindrical", "main-pulsar2d-cylindrical.cpp", None, CYL,
           "cyl_pulsar_fields"),
    # the same programs built without EZ: the staggered solver field_solver
    Driver("wave-yee", "main-wave.cpp", 0, YEE, "alfven_plane_wave_fields"),
    Driver("pulsar3d-yee", "main-pulsar3d.cpp", 1, YEE, "pulsar_fields"),
    Driver("alfven3d-yee", "main-alfven3d.cpp", 2, YEE, "pulsar_fields"),
    Driver("gr-yee", "main-gr-Yee.cpp", None, GRYEE, "wald_fields"),
)}


def parse_args(argv=None):
    ap = argparse.ArgumentParser(prog="python -m coffee_b200",
                                 description="Run a COFFEE driver on the B200 library.")
    ap.add_argument("driver", choices=sorted(DRIVERS))
    ap.add_argument("-c", "--config", default="config.toml", help="the reference's config.toml")
    ap.add_argument("-o", "--output", default="Data", help="output directory")
    ap.add_argument("--restart", default=None, help="snapshot file to continue from")
    ap.add_argument("--steps", type=int, default=None, help="override max_steps")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--precision", choices=("f32", "f64"), default="f32")
    ap.add_argument("--energy-diag", action="store_true",
                    help="flat drivers: write the CPU build's dU_* energy diagnostics")
    return ap.parse_args(argv)


def plan(args) -> tuple[Driver, SimParams]:
    """The driver and its parameters; raises ValueError where the reference
    program would abort (wrong problem id)."""
    d = DRIVERS[args.driver]
    p = SimParams.from_toml(args.config)
    if args.steps is not None:
        p.max_steps = int(args.steps)
    if d.problem is not None and p.problem != d.problem:
        raise ValueError(f"{d.program} solves problem {d.problem}; set 'problem' to "
                         f"{d.problem} in {args.config} (it is {p.problem})")
    return d, p


def events(max_steps: int, data_interval: int, snapshot_interval: int, start: int = 0,
           restarted: bool = False):
    """(step, output, snapshot) for every step of the loop from `start` to
    max_steps at which the reference's loop writes something; after a
    restart nothing is written at the restart step itself
    (``step != prev_snapshot``)."""
    out = []
    for step in range(start, max_steps + 1):
        o = data_interval > 0 and step % data_interval == 0
        s = snapshot_interval > 0 and step % snapshot_interval == 0
        if restarted and step == start:
            o = s = False
        if o or s:
            out.append((step, o, s))
    return out


def _solver(kind, data, env, sem_gpu):
    from . import solver as sv
    if kind == FLAT:
        return sv.FieldSolverEZ(data, env, "gpu" if sem_gpu else "cpu")
    return {GR: sv.FieldSolverGrEZ, SPH: sv.FieldSolverEZSpherical,
            CYL: sv.FieldSolverEZCylindrical, YEE: sv.FieldSolver,
            GRYEE: sv.FieldSolverGr}[kind](data, env)


def _write_output(path, data, s, step, time, ds, guard, flat, energy_diag=False):
    names = ["Ex", "Ey", "Ez", "Bx", "By", "Bz", "P"]
    arrays = data.download(names)
    if flat:
        arrays += data.download(["Jx", "Jy", "Jz", "divE", "divB"])
        names += ["Jx", "Jy", "Jz", "divE", "divB"]
    if energy_diag:
        from ._lib import ENERGY_DIAG_NAMES, FIELD_IDS
        arrays += data.download(ENERGY_DIAG_NAMES)
        zero = np.zeros_like(arrays[0])
        for name in ENERGY_DIAG_NAMES[3:]:
            data.upload_field(FIELD_IDS[name], zero)
    sl = tuple(slice(g, a - g, ds) for g, a in zip(guard[::-1], arrays[0].shape))
    write_fld(path, [np.ascontiguousarray(a[sl]) for a in arrays], guard=(0, 0, 0), time=time,
              step=step)


def run(args) -> int:
    from .solver import SimData, SimEnvironment

    d, p = plan(args)
    dtype = np.float32 if args.precision == "f32" else np.float64
    os.makedirs(args.output, exist_ok=True)
    env = SimEnvironment(p, device=args.device)
    data = SimData(env, dtype)
    init = getattr(problems, d.init)
    data.upload(init(p, dtype, yee=True) if d.kind in (YEE, GRYEE) else init(p, dtype))
    flat = d.kind == FLAT
    energies = d.kind in (FLAT, YEE)
    s = _solver(d.kind, data, env, sem_gpu=False)
    if flat:
        s.set_aux(True)  # J, div E, div B for the outputs
    energy_diag = bool(getattr(args, "energy_diag", False))
    if energy_diag:
        if not flat:
            raise ValueError("--energy-diag needs a flat (field_solver_EZ) driver")
        s.set_energy_diag(True)
    ftype = np.dtype(dtype).type
    dt = ftype(p.dt)
    step, time = 0, ftype(0.0)
    if args.restart:
        t0, step = s.load_snapshot(args.restart)
        time = ftype(t0)
    guard = tuple(p.guard)
    ds = max(1, int(p.downsample))
    for ev_step, out, snap in events(p.max_steps, p.data_interval, p.snapshot_interval, step,
                                     restarted=bool(args.restart)):
        n = ev_step - step
        if n > 0:
            s.step(float(time), n)
            for _ in range(n):
                time = ftype(time + dt)
            step = ev_step
        if snap:
            s.save_snapshot(os.path.join(args.output, f"snapshot.{step:05d}.fld"), float(time),
                            step)
        if out:
            _write_output(os.path.join(args.output, f"fld.{step:05d}.fld"), data, s, step,
                          float(time), ds, guard, flat, energy_diag)
            if energies:
                wb, we = s.total_energy("B"), s.total_energy("E")
                with open(os.path.join(args.output, "energy.txt"), "a") as fh:
                    fh.write(f"{step} {float(time):.9g} {wb:.17g} {we:.17g}\n")
        print(f"step = {step}", flush=True)
    # the loop's last evolve_fields runs after the output of step max_steps
    if step <= p.max_steps:
        n = p.max_steps + 1 - step
        s.step(float(time), n)
        for _ in range(n):
            time = ftype(time + dt)
        step = p.max_steps + 1
    print(f"done: {step} evolve_fields calls, time = {float(time):.9g}", flush=True)
    s.close()
    data.close()
    env.close()
    return 0


def main(argv=None) -> int:
    args = parse_args(argv)
    try:
        return run(args)
    except ValueError as e:
        print(f"error: {e}", file=sys.stderr)
        return 2
