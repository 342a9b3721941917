"""The oracle restatement (oracle/ffe_oracle.c) pinned against the
reference's own CPU build, through the committed golden fixtures
(tests/golden/*.npz, made by tests/golden/make_golden.py from oracle/_ref)."""
import numpy as np
import pytest

from helpers import (count_differing, fp32_parity, golden_cases, load_golden, rel_l2,
                     wide_box_case)
from oracle import oracle


# Fixtures without the rotating star or an absorbing layer: there the
# restatement follows the reference CPU build's arithmetic operation for
# operation (the products its compiler fuses into FMAs, its vector library's
# tanh), so it reproduces the float and the double build bit for bit.
EXACT_CASES = ("alfven16", "noclean16", "turb16")


@pytest.mark.parametrize("name", EXACT_CASES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_port_is_the_reference_bit_for_bit(name, dtype):
    p, d = load_golden(name)
    lanes = 16 if dtype == np.float32 else 8
    out, _ = oracle.run_port(p, [a.astype(dtype) for a in d["in_f32"]], int(d["steps"]),
                             time0=float(d["time0"]), taper_lanes=lanes)
    ref = d["out_f32"] if dtype == np.float32 else d["out_f64"]
    for f in range(7):
        diff = int(np.count_nonzero(out[f] != ref[f]))
        assert diff == 0, (name, f, diff, rel_l2(out[f], ref[f]))


@pytest.mark.parametrize("name", golden_cases())
def test_port_matches_reference_fp64(name):
    p, d = load_golden(name)
    f64 = [a.astype(np.float64) for a in d["in_f32"]]
    out, _ = oracle.run_port(p, f64, int(d["steps"]), time0=float(d["time0"]), taper_lanes=8)
    for f in range(7):
        assert rel_l2(out[f], d["out_f64"][f]) < 1e-11, (name, f)


@pytest.mark.parametrize("name", golden_cases())
def test_port_matches_reference_fp32(name):
    p, d = load_golden(name)
    aux = "aux_f32" in d
    out, auxo = oracle.run_port(p, list(d["in_f32"]), int(d["steps"]), time0=float(d["time0"]),
                                taper_lanes=16, aux=aux)
    ok, rep = fp32_parity(out, d["out_f32"], d["out_f64_l16"])
    assert ok, rep
    if aux:
        g = p.guard
        sl = tuple(slice(g[a], g[a] + p.N[a]) for a in (2, 1, 0))
        for f in range(5):
            assert rel_l2(auxo[f][sl], d["aux_f32"][f][sl]) < 1e-4, (name, f)


def test_fp64_same_algorithm_fixture_is_the_port():
    # out_f64_l16 of a fixture is the port in FP64 with 16 taper lanes
    p, d = load_golden("alfven16")
    f64 = [a.astype(np.float64) for a in d["in_f32"]]
    out, _ = oracle.run_port(p, f64, int(d["steps"]), taper_lanes=16)
    for f in range(7):
        assert np.array_equal(out[f], d["out_f64_l16"][f])


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_port_matches_reference_shifted_box():
    """A fresh case straight from the reference binary (not a fixture):
    non-cubic periodic box, no E.B damping."""
    from coffee_b200 import problems

    p = problems.alfven_params(16)
    p.N = [32, 16, 16]
    p.size = [2.0, 1.0, 1.0]
    p.use_edotb_damping = False
    f32 = problems.alfven_fields(p, np.float32)
    f64 = [a.astype(np.float64) for a in f32]
    ref, _, _ = oracle.run_reference(p, f64, 3)
    out, _ = oracle.run_port(p, f64, 3, taper_lanes=8)
    for f in range(7):
        assert rel_l2(out[f], ref[f]) < 1e-11


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_port_is_the_reference_across_the_taper():
    """A fresh case from the reference float build itself: a box around the
    origin where the taper's tanh takes both of its branches."""
    p, f32 = wide_box_case()
    ref, _, _ = oracle.run_reference(p, f32, 3)
    out, _ = oracle.run_port(p, f32, 3, taper_lanes=16)
    for f in range(7):
        assert count_differing(out[f], ref[f]) == 0, (f, rel_l2(out[f], ref[f]))


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["alfven16", "turb16", "wide"])
def test_port_energy_diagnostics_are_the_reference(name):
    """The CPU build's energy-change arrays (dU_EgtB, dU_Epar, dU_KO and the
    _cum sums, the latter from zero) after 3 steps, bit for bit on the
    interior, from the reference float build itself."""
    if name == "wide":
        p, f32 = wide_box_case()
    else:
        p, d = load_golden(name)
        f32 = list(d["in_f32"])
    _, _, info = oracle.run_reference(p, f32, 3, diag=True)
    dg = [np.zeros_like(f32[0]) for _ in range(6)]
    oracle.run_port(p, f32, 3, taper_lanes=16, diag=dg)
    g = p.guard
    sl = tuple(slice(g[a], g[a] + p.N[a]) for a in (2, 1, 0))
    for k in range(6):
        assert count_differing(dg[k][sl], info["diag"][k][sl]) == 0, (name, k)
    assert float(np.abs(info["diag"][2][sl]).max()) > 0
