"""The GR and log-spherical configurations at their stated size and length,
against the reference's own GPU build (oracle/_ref/coffee_refgpu_float and
_double, compiled from the reference's sources).

These runs take minutes each on a B200 (most of it in the reference's own
build), so they run only when COFFEE_LONG_RUNS=1 is set:

    COFFEE_LONG_RUNS=1 python -m pytest tests/test_long_configs.py -m gpu -s

* GR Kerr-Schild Wald problem: 256^3 + 3 guards, a = 0.9, M = 1, [-20, 20]^3,
  absorbing layer 16 cells, B = z / sqrt(gamma), D = 0 (the reference's
  user_wald2.hpp), 2000 steps (the loop of main-gr.cpp) with the reference's
  inner absorbing region.
* Log-spherical aligned dipole (r in [1, 100], theta in [0, pi]) on each of
  the configuration's grid sizes 512x256, 768x384, 1024x512, 2048x1024, for
  5 rotation periods at R_LC = 3 (the fastest spin of the configuration's
  range [3, 10], hence the fewest steps: 5 * 2 pi / (Omega dt)).

Each FP32 result of the library must sit within the bar of
helpers.fp32_parity of the reference float build, the FP32 noise being the
float build's distance from the same algorithm in FP64.  The FP64 run is the
library's own FP64 mode (pinned to the reference double build at small
sizes by tests/test_gpu_variants.py); for the GR case the reference double
build is also run, and the library's FP64 result must lie within 5% of the
float build's distance from it.  The per-field errors are printed.
"""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from coffee_b200 import problems
from coffee_b200.solver import FieldSolverEZSpherical, FieldSolverGrEZ, SimData, SimEnvironment
from helpers import fp32_parity, rel_l2
from oracle import oracle

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(os.environ.get("COFFEE_LONG_RUNS") != "1",
                       reason="long configurations run only with COFFEE_LONG_RUNS=1"),
]


def _run_ours(cls, p, fields, nsteps, dtype):
    env = SimEnvironment(p)
    data = SimData(env, dtype)
    data.upload([a.astype(dtype) for a in fields])
    solver = cls(data, env)
    solver.step(0.0, nsteps)
    solver.check_finite()
    out = data.download()
    solver.close()
    data.close()
    env.close()
    return out


def _report(tag, out, r32, r64, extra=None):
    ok, rep = fp32_parity(out, r32, r64)
    print(f"--- {tag}\n{rep}")
    if extra:
        print(extra)
    return ok, rep


def test_gr_wald256_2000_steps():
    p = problems.wald_params(N=256, half_size=20.0, a=0.9, pml=16)
    nsteps = 2000
    f64 = problems.wald_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    ref32, _, info32 = oracle.run_reference_gpu("gr", p, f32, nsteps, timeout=3000)
    ref64, _, info64 = oracle.run_reference_gpu("gr", p, f64, nsteps, timeout=6000)
    out32 = _run_ours(FieldSolverGrEZ, p, f32, nsteps, np.float32)
    out64 = _run_ours(FieldSolverGrEZ, p, f64, nsteps, np.float64)
    extra = "library FP64 vs reference double build: " + ", ".join(
        f"{rel_l2(out64[f], ref64[f]):.1e}" for f in range(7))
    ok, rep = _report("GR Wald 256^3, 2000 steps", out32, ref32, ref64, extra)
    assert ok, rep
    # two FP64 evaluations of the same scheme part where a clamp or an
    # absorbing-region test flips on a last-bit difference, and near the
    # horizon such differences grow; they must stay far below the float
    # build's own distance from the double build
    for f in range(7):
        noise = rel_l2(ref32[f], ref64[f])
        assert rel_l2(out64[f], ref64[f]) <= 0.05 * noise, (f, extra)


@pytest.mark.parametrize("nr,nth", [(512, 256), (768, 384), (1024, 512), (2048, 1024)])
def test_logsph_five_periods(nr, nth):
    r_lc = 3.0
    p = problems.sph_pulsar_params(nr=nr, nth=nth, guard=4, omega=1.0 / r_lc)
    nsteps = int(math.ceil(5 * 2 * math.pi / (p.omega * p.dt)))
    f64 = problems.sph_pulsar_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    ref32, _, _ = oracle.run_reference_gpu("sph", p, f32, nsteps, timeout=3000)
    out32 = _run_ours(FieldSolverEZSpherical, p, f32, nsteps, np.float32)
    out64 = _run_ours(FieldSolverEZSpherical, p, f64, nsteps, np.float64)
    ok, rep = _report(f"log-spherical {nr}x{nth}, R_LC = {r_lc}, {nsteps} steps (5 periods)",
                      out32, ref32, out64)
    assert ok, rep
