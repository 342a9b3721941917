"""Parity of the log-spherical, cylindrical and GR (Kerr-Schild) solvers
with the reference's own GPU build (oracle/_ref/coffee_refgpu_*, compiled
from the reference's field_solver_EZ_spherical.cu,
field_solver_EZ_cylindrical.cu and field_solver_gr_EZ.cu), which is the only
build the reference has of these solvers.

Each case runs the same input through the reference's float and double
builds and through coffee_b200 in FP32; the FP32 result must sit within the
float build's own distance from the double build (tests/helpers.fp32_parity).
The numpy restatements (oracle/axisym_oracle.py, oracle/gr_oracle.py) are
checked against the double build in the same runs.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from coffee_b200 import problems
from coffee_b200._lib import COFFEE_E_TIMEOUT, CoffeeError
from coffee_b200.solver import FieldSolverEZCylindrical, FieldSolverEZSpherical, \
    FieldSolverGrEZ, SimData, SimEnvironment, SphBatch
from helpers import fp32_parity, rel_l2
from oracle import axisym_oracle as axo
from oracle import gr_oracle
from oracle import oracle

pytestmark = pytest.mark.gpu


def _need_refgpu():
    for dt in (np.float32, np.float64):
        if not os.path.exists(oracle.refgpu_binary(dt)):
            pytest.fail(f"{oracle.refgpu_binary(dt)} missing: build it with `make -C oracle gpuref REF=<reference checkout>`")


def _run_ours(cls, p, fields32, nsteps, aux=False, dtype=np.float32):
    env = SimEnvironment(p)
    data = SimData(env, dtype)
    data.upload(fields32)
    solver = cls(data, env)
    if aux:
        solver.set_aux(True)
    solver.step(0.0, nsteps)
    out = data.download()
    auxo = data.download(("Jx", "Jy", "Jz", "divE", "divB")) if aux else None
    solver.close()
    data.close()
    env.close()
    return out, auxo


def _compare(tag, out, r32, r64, np64=None):
    ok, rep = fp32_parity(out, r32, r64)
    print(f"--- {tag}\n{rep}")
    assert ok, f"{tag}: FP32 parity with the reference GPU build failed\n{rep}"
    if np64 is not None:
        worst = max(rel_l2(np64[f], r64[f]) for f in range(7))
        print(f"numpy restatement vs reference double build: {worst:.2e}")
        assert worst < 1e-9, f"{tag}: numpy restatement departs from the reference ({worst:.2e})"


SPH_CASES = {
    # dipole star with a spin perturbation, absorbing layer, geometric KO
    "sph_pulsar": dict(),
    # plain KO, E.B damping in the current, one shifted ghost layer
    "sph_plainko_edotb_shift": dict(KO_geometry=False, use_edotb_damping=True, shift_ghost=1),
}


@pytest.mark.parametrize("case", sorted(SPH_CASES))
def test_logsph_matches_reference_gpu_build(case):
    _need_refgpu()
    p = problems.sph_pulsar_params(nr=64, nth=32, guard=4, omega=0.25)
    p.tp_start, p.tp_end, p.dw0, p.thp1, p.thp2 = 0.0, 0.5, 0.1, 0.6, 1.2
    for k, v in SPH_CASES[case].items():
        setattr(p, k, v)
    nsteps = 24
    f64 = problems.sph_pulsar_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    r64, _, _ = oracle.run_reference_gpu("sph", p, f64, nsteps)
    r32, _, _ = oracle.run_reference_gpu("sph", p, f32, nsteps)
    np64 = axo.sph_evolve(p, np.stack([a[0] for a in f64]), nsteps)
    out, _ = _run_ours(FieldSolverEZSpherical, p, f32, nsteps)
    _compare(case, out, r32, r64, [a[None] for a in np64])


CYL_CASES = {
    "cyl_pulsar": dict(),
    "cyl_noclamps": dict(clean_ep=False, check_egb=False, KOeps=0.3),
}


@pytest.mark.parametrize("case", sorted(CYL_CASES))
def test_cylindrical_matches_reference_gpu_build(case):
    _need_refgpu()
    p = problems.cyl_pulsar_params(nR=64, nz=128, guard=3)
    p.tp_start, p.tp_end, p.dw0, p.rpert1, p.rpert2 = 0.0, 2.0, 0.05, 3.0, 6.0
    for k, v in CYL_CASES[case].items():
        setattr(p, k, v)
    nsteps = 24
    f64 = problems.cyl_pulsar_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    r64, _, _ = oracle.run_reference_gpu("cyl", p, f64, nsteps)
    r32, _, _ = oracle.run_reference_gpu("cyl", p, f32, nsteps)
    np64 = axo.cyl_evolve(p, np.stack([a[0] for a in f64]), nsteps)
    out, _ = _run_ours(FieldSolverEZCylindrical, p, f32, nsteps)
    _compare(case, out, r32, r64, [a[None] for a in np64])


GR_CASES = {
    # Wald field around a spin-0.9 hole: outer and inner absorbing layers
    "gr_wald": dict(),
    # without the divergence cleaning terms, one shifted ghost layer
    "gr_wald_noclean_shift": dict(divB_clean=False, shift_ghost=1, guard=[4, 4, 4]),
}


@pytest.mark.parametrize("case", sorted(GR_CASES))
def test_gr_matches_reference_gpu_build(case):
    _need_refgpu()
    p = problems.wald_params(N=40, half_size=5.0, a=0.9, pml=6)
    for k, v in GR_CASES[case].items():
        setattr(p, k, v)
    nsteps = 16
    f64 = problems.wald_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    r64, _, _ = oracle.run_reference_gpu("gr", p, f64, nsteps)
    r32, _, _ = oracle.run_reference_gpu("gr", p, f32, nsteps)
    np64 = gr_oracle.gr_evolve(p, np.stack(f64), nsteps)
    out, _ = _run_ours(FieldSolverGrEZ, p, f32, nsteps)
    _compare(case, out, r32, r64, list(np64))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gr_eh_from_the_writing_kernel_is_bitwise(dtype, monkeypatch):
    """E and H written by the stage and KO kernels for the next kernel (with
    one E, H pass per call) give bitwise the fields of an E, H pass before
    every stage, over calls of several steps and single steps, with the
    inner and outer absorbing layers active."""
    p = problems.wald_params(N=40, half_size=5.0, a=0.9, pml=6)
    f = [a.astype(dtype) for a in problems.wald_fields(p, np.float64)]

    def run(per_stage):
        monkeypatch.setenv("COFFEE_GR_EH_PER_STAGE", "1" if per_stage else "0")
        env = SimEnvironment(p)
        data = SimData(env, dtype)
        data.upload(f)
        solver = FieldSolverGrEZ(data, env)
        solver.step(0.0, 5)
        solver.step(0.0, 1)
        solver.step(0.0, 3)
        out = data.download()
        solver.close()
        data.close()
        env.close()
        return out

    a, b = run(False), run(True)
    for k in range(7):
        assert np.array_equal(a[k], b[k]), k


def test_gr_tiled_stage_is_bitwise(monkeypatch):
    """The FP32 stage streamed through shared-memory tiles gives bitwise the
    fields of the per-point stage kernel: an 80^3 Wald run (two z chunks of
    the tiled kernel, a ragged last one), both absorbing layers, the
    near-horizon metric table, over several calls."""
    p = problems.wald_params(N=80, half_size=10.0, a=0.9, pml=8)
    f = [a.astype(np.float32) for a in problems.wald_fields(p, np.float64)]

    def run(untiled):
        monkeypatch.setenv("COFFEE_GR_TILED", "0" if untiled else "1")
        env = SimEnvironment(p)
        data = SimData(env, np.float32)
        data.upload(f)
        solver = FieldSolverGrEZ(data, env)
        solver.set_aux(True)
        solver.step(0.0, 3)
        solver.step(0.0, 2)
        out = data.download()
        aux = data.download(("Jx", "Jy", "Jz", "divE", "divB"))
        solver.close()
        data.close()
        env.close()
        return out, aux

    (a, xa), (b, xb) = run(False), run(True)
    for k in range(7):
        assert np.array_equal(a[k], b[k]), k
    for k in range(5):
        assert np.array_equal(xa[k], xb[k]), ("aux", k)


FLAT_CASES = {
    "flat_pulsar": lambda: problems.pulsar_params(N=40, guard=3, half_size=10.0, radius=2.5,
                                                  omega=0.1, pml=6),
    "flat_alfven_periodic": lambda: problems.alfven_params(N=32, guard=3),
}


@pytest.mark.parametrize("case", sorted(FLAT_CASES))
def test_flat_gpu_semantics_matches_reference_gpu_build(case):
    """COFFEE_SEM_GPU_REF against the reference's own field_solver_EZ.cu."""
    from coffee_b200.solver import run_flat
    _need_refgpu()
    p = FLAT_CASES[case]()
    nsteps = 12
    if p.problem == 0:
        f64 = problems.alfven_fields(p, np.float64)
    else:
        f64 = problems.pulsar_fields(p, np.float64)
    f32 = [a.astype(np.float32) for a in f64]
    r64, _, _ = oracle.run_reference_gpu("ez", p, f64, nsteps)
    r32, _, _ = oracle.run_reference_gpu("ez", p, f32, nsteps)
    out, _ = run_flat(p, f32, nsteps, semantics="gpu")
    _compare(case, out, r32, r64)


def test_logsph_rejects_short_theta_guard():
    """guard[1] = 3 with theta reaching pi: the reference's axis boundary
    would write past the array; the library refuses the configuration."""
    p = problems.sph_pulsar_params(nr=32, nth=16, guard=4)
    p.guard = [4, 3, 0]
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    with pytest.raises(RuntimeError, match="guard"):
        FieldSolverEZSpherical(data, env)


def _batch_runs(dtype, nsteps=7):
    """Three log-spherical runs of different sizes, spins and layers: their
    single-run results after nsteps steps, their initial fields, and a
    (env, data, solver) of each for a batch."""
    cfgs = [dict(nr=64, nth=32, omega=0.2, pml=8), dict(nr=96, nth=48, omega=0.3, pml=0),
            dict(nr=48, nth=24, omega=0.1, pml=6)]
    singles, inits, runs = [], [], []
    for k, cfg in enumerate(cfgs):
        p = problems.sph_pulsar_params(guard=4, **cfg)
        if k == 0:
            p.tp_start, p.tp_end, p.dw0, p.thp1, p.thp2 = 0.0, 0.5, 0.1, 0.6, 1.2
        f = problems.sph_pulsar_fields(p, dtype)
        out, _ = _run_ours(FieldSolverEZSpherical, p, f, nsteps, dtype=dtype)
        singles.append(out)
        inits.append(f)
        env = SimEnvironment(p)
        data = SimData(env, dtype)
        data.upload(f)
        runs.append((env, data, FieldSolverEZSpherical(data, env)))
    return singles, inits, runs


def _check_batch(runs, singles):
    for k, (env, data, solver) in enumerate(runs):
        got = data.download()
        for f in range(7):
            assert np.array_equal(got[f], singles[k][f]), f"run {k} field {f} differs"


def _close_runs(batch, runs):
    batch.close()
    for env, data, solver in runs:
        solver.close()
        data.close()
        env.close()


def test_logsph_batch_equals_single_runs():
    """One launch per phase over runs of different sizes, spins and layers
    gives bitwise the results of stepping each run alone."""
    singles, _, runs = _batch_runs(np.float32)
    batch = SphBatch([r[2] for r in runs])
    info = batch.info()  # the autotuner's choice: any candidate gives the same fields
    assert info["tile"] in ([32, 8], [64, 4], [128, 2], [16, 16]) and info["first_stage_ms"] > 0
    batch.step(3)  # captures the step graph, replays it 3 times
    batch.step(4)  # replays it from the new times
    _check_batch(runs, singles)
    _close_runs(batch, runs)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_logsph_persistent_batch_equals_single_runs(dtype):
    """The persistent mode (one cooperative launch per call, grid-wide
    barriers between the phases) gives bitwise the single runs' results."""
    singles, _, runs = _batch_runs(dtype)
    batch = SphBatch([r[2] for r in runs])
    batch.set_persistent(True)
    batch.step(3)
    batch.step(4)
    _check_batch(runs, singles)
    _close_runs(batch, runs)


def test_logsph_persistent_batch_wait_limit():
    """A barrier wait that runs out ends the persistent launch with
    COFFEE_E_TIMEOUT (one CTA leaves out its first arrival, so the others
    wait for it until the 1 ms limit); the context stays usable and the next
    calls, from the initial fields again, give the single runs' results."""
    singles, inits, runs = _batch_runs(np.float32)
    batch = SphBatch([r[2] for r in runs])
    batch.set_persistent(True)
    batch.set_wait_limit(1_000_000, stall_block=0)
    with pytest.raises(CoffeeError) as err:
        batch.step(2)
    assert err.value.code == COFFEE_E_TIMEOUT and "grid barrier 0" in str(err.value)
    batch.set_wait_limit(2_000_000_000, stall_block=-1)
    for (env, data, solver), f in zip(runs, inits):
        data.upload(f)
    batch.times[:] = 0.0
    batch.step(7)
    _check_batch(runs, singles)
    _close_runs(batch, runs)
