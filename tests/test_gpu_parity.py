"""Parity of the CUDA field update (through the C ABI) with the oracle.

In its default arithmetic the FP32 CPU-semantics solver computes every
operation of the reference float build in that build's order and rounding,
so where no star or absorbing layer acts its fields must equal the float
build's bit for bit (0 differing points).  Everything else in FP32 (the star
and absorbing boundaries, the GPU semantics, the fast arithmetic) is held to
the bar of helpers.fp32_parity: within max(2e-5, 4 x noise) relative L2 of
the reference float build, per field, where `noise` is the float build's own
distance from the same algorithm in FP64, and no less accurate than the
float build against that FP64 run (up to 2x + 2e-5).  FP64 results must
match the reference FP64 build to 1e-10.
"""
import numpy as np
import pytest

from coffee_b200 import problems
from coffee_b200.solver import run_flat
from helpers import (count_differing, fp32_parity, golden_cases, interior, load_golden,
                     rel_l2, wide_box_case)
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_cases())
def test_golden_fp32(name):
    p, d = load_golden(name)
    aux = "aux_f32" in d
    out, auxo = run_flat(p, list(d["in_f32"]), int(d["steps"]), time0=float(d["time0"]),
                         semantics="cpu", aux=aux)
    ok, rep = fp32_parity(out, d["out_f32"], d["out_f64_l16"])
    assert ok, rep
    if aux:
        sl = interior(p)
        for f in range(5):
            assert rel_l2(auxo[f][sl], d["aux_f32"][f][sl]) < 2e-4, (name, f)


EXACT_CASES = ("alfven16", "noclean16", "turb16")


@pytest.mark.parametrize("name", EXACT_CASES)
def test_golden_fp32_bit_for_bit(name):
    """The float build's fields, J, divE and divB, bit for bit."""
    p, d = load_golden(name)
    aux = "aux_f32" in d
    out, auxo = run_flat(p, list(d["in_f32"]), int(d["steps"]), time0=float(d["time0"]),
                         semantics="cpu", aux=aux)
    for f in range(7):
        assert count_differing(out[f], d["out_f32"][f]) == 0, \
            (name, f, rel_l2(out[f], d["out_f32"][f]))
    if aux:
        sl = interior(p)
        for f in range(5):
            assert count_differing(auxo[f][sl], d["aux_f32"][f][sl]) == 0, (name, "aux", f)


@pytest.mark.parametrize("name", golden_cases())
def test_golden_fp32_fast_arithmetic(name):
    p, d = load_golden(name)
    out, _ = run_flat(p, list(d["in_f32"]), int(d["steps"]), time0=float(d["time0"]),
                      semantics="cpu", arithmetic="fast")
    ok, rep = fp32_parity(out, d["out_f32"], d["out_f64_l16"])
    assert ok, rep


def test_wide_box_bit_for_bit():
    """Both branches of the taper's tanh (a box around the origin) against
    the restatement, which equals the reference float build bit for bit
    (tests/test_oracle.py), and against that build where it is built."""
    p, f32 = wide_box_case()
    out, _ = run_flat(p, f32, 3)
    ref, _ = oracle.run_port(p, f32, 3, taper_lanes=16)
    for f in range(7):
        assert count_differing(out[f], ref[f]) == 0, (f, rel_l2(out[f], ref[f]))
    if oracle.reference_available(np.float32):
        refb, _, _ = oracle.run_reference(p, f32, 3)
        for f in range(7):
            assert count_differing(out[f], refb[f]) == 0, f


@pytest.mark.parametrize("name", golden_cases())
def test_golden_fp64(name):
    p, d = load_golden(name)
    f64 = [a.astype(np.float64) for a in d["in_f32"]]
    out, _ = run_flat(p, f64, int(d["steps"]), time0=float(d["time0"]), semantics="cpu")
    for f in range(7):
        assert rel_l2(out[f], d["out_f64"][f]) < 1e-10, (name, f, rel_l2(out[f], d["out_f64"][f]))


def _check_vs_port(p, f32, steps, semantics, t0=0.0):
    sem = oracle.SEM_CPU_REF if semantics == "cpu" else oracle.SEM_GPU_REF
    ref32, _ = oracle.run_port(p, f32, steps, time0=t0, semantics=sem, taper_lanes=16)
    ref64, _ = oracle.run_port(p, [a.astype(np.float64) for a in f32], steps, time0=t0,
                               semantics=sem, taper_lanes=16)
    out, _ = run_flat(p, f32, steps, time0=t0, semantics=semantics)
    ok, rep = fp32_parity(out, ref32, ref64)
    assert ok, rep
    # guard points hold exactly what the kernels wrote: compare them too
    for f in range(7):
        assert rel_l2(out[f], ref32[f]) <= max(1e-4, 8 * rel_l2(ref32[f], ref64[f])), f


@pytest.mark.parametrize("semantics", ["cpu", "gpu"])
def test_alfven_both_semantics(semantics):
    p = problems.alfven_params(32)
    _check_vs_port(p, problems.alfven_fields(p, np.float32), 6, semantics)


@pytest.mark.parametrize("semantics", ["cpu", "gpu"])
def test_pulsar_absorbing_both_semantics(semantics):
    p = problems.pulsar_params(N=32, half_size=8.0, radius=2.0, omega=0.1, b0=1.0, pml=6)
    p.q11 = 0.05
    p.q12 = 0.02
    p.p1 = 0.3
    _check_vs_port(p, problems.pulsar_fields(p, np.float32), 4, semantics, t0=0.3)


def test_mixed_boundaries_noncubic():
    p = problems.turbulence_params(16)
    p.N = [48, 16, 32]
    p.size = [3.0, 1.0, 2.0]
    p.periodic_boundary = [True, False, True]
    p.pml = [0, 3, 0]
    p.pmllen = 2
    _check_vs_port(p, problems.turbulence_fields(p, np.float32), 5, "cpu")


def test_shift_ghost():
    p = problems.alfven_params(16)
    p.guard = [5, 5, 5]
    p.shift_ghost = 2
    p.periodic_boundary = [True, False, True]
    _check_vs_port(p, problems.alfven_fields(p, np.float32), 3, "gpu")


def test_no_cleaning_no_damping():
    p = problems.turbulence_params(32)
    p.divB_clean = False
    p.use_edotb_damping = False
    p.KOeps = 0.1
    p.clean_ep = False
    p.check_egb = False
    for sem in ("cpu", "gpu"):
        _check_vs_port(p, problems.turbulence_fields(p, np.float32), 4, sem)


def test_config1_alfven128_100_steps():
    """The Alfven-wave configuration at full size and length: 128^3 + 3
    guards, periodic, dt = dx/2, 100 steps, all 7 fields, against the
    reference float build when it is built here (else the restatement, which
    equals it bit for bit): every field within the stated bound of 1e-5
    relative L2, and in fact bit for bit.  The error against the same
    algorithm in FP64 is reported."""
    p = problems.alfven_params(128)
    f32 = problems.alfven_fields(p, np.float32)
    if oracle.reference_available(np.float32):
        ref32, _, _ = oracle.run_reference(p, f32, 100)
    else:
        ref32, _ = oracle.run_port(p, f32, 100, taper_lanes=16)
    ref64, _ = oracle.run_port(p, [a.astype(np.float64) for a in f32], 100, taper_lanes=16)
    out, _ = run_flat(p, f32, 100)
    for f in range(7):
        e32, e64 = rel_l2(out[f], ref32[f]), rel_l2(out[f], ref64[f])
        print(f"field {f}: vs float build {e32:.2e}, vs FP64 {e64:.2e}, "
              f"differing points {count_differing(out[f], ref32[f])}")
        assert e32 <= 1e-5, (f, e32)
        assert count_differing(out[f], ref32[f]) == 0, f


def test_config1_fast_arithmetic():
    """The same configuration in the regrouped (fast) arithmetic: within the
    FP32 noise bar of the reference float build."""
    p = problems.alfven_params(128)
    f32 = problems.alfven_fields(p, np.float32)
    ref32, _ = oracle.run_port(p, f32, 100, taper_lanes=16)
    ref64, _ = oracle.run_port(p, [a.astype(np.float64) for a in f32], 100, taper_lanes=16)
    out, _ = run_flat(p, f32, 100, arithmetic="fast")
    ok, rep = fp32_parity(out, ref32, ref64)
    print(rep)
    assert ok, rep


@pytest.mark.parametrize("name", ["alfven16", "turb16", "wide"])
def test_energy_diagnostics_bit_for_bit(name):
    """The CPU build's energy-change diagnostics (dU_EgtB, dU_Epar, dU_KO and
    the _cum sums from zero) after 3 steps: against the restatement (itself
    bit for bit the reference float build, tests/test_oracle.py) and against
    the reference where it is built, bit for bit on the interior."""
    if name == "wide":
        p, f32 = wide_box_case()
    else:
        p, d = load_golden(name)
        f32 = list(d["in_f32"])
    out, extra = run_flat(p, f32, 3, energy_diag=True)
    dg = [np.zeros_like(f32[0]) for _ in range(6)]
    ref, _ = oracle.run_port(p, f32, 3, taper_lanes=16, diag=dg)
    sl = interior(p)
    for f in range(7):
        assert count_differing(out[f], ref[f]) == 0, (name, f)
    for k in range(6):
        assert count_differing(extra[k][sl], dg[k][sl]) == 0, (name, "dU", k)
    if oracle.reference_available(np.float32):
        _, _, info = oracle.run_reference(p, f32, 3, diag=True)
        for k in range(6):
            assert count_differing(extra[k][sl], info["diag"][k][sl]) == 0, (name, "ref dU", k)


def test_fp64_with_the_float_builds_taper_lanes():
    """FP64 with the float build's 16 taper lanes (coffee_solver_set_taper_lanes)
    is the float build's algorithm without FP32 rounding: it matches the
    restatement in FP64 with 16 lanes (the fixtures' out_f64_l16)."""
    from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment
    p, d = load_golden("alfven16")
    env = SimEnvironment(p)
    data = SimData(env, np.float64)
    data.upload([a.astype(np.float64) for a in d["in_f32"]])
    s = FieldSolverEZ(data, env, "cpu")
    s.set_taper_lanes(16)
    s.step(float(d["time0"]), int(d["steps"]))
    out = data.download()
    s.close()
    data.close()
    env.close()
    for f in range(7):
        assert rel_l2(out[f], d["out_f64_l16"][f]) < 1e-12, f
