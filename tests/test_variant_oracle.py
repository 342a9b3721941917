"""The numpy restatements of the reference's log-spherical, cylindrical, GR
and staggered solvers (oracle/axisym_oracle.py, oracle/gr_oracle.py,
oracle/yee_oracle.py) against fixtures
made by the reference's own GPU build in double precision
(tests/golden/variants/*.npz, written by tests/golden/make_variant_golden.py
on a GPU).  CPU only."""
from __future__ import annotations

import glob
import importlib.util
import os

import numpy as np
import pytest

from helpers import GOLDEN, rel_l2
from oracle import axisym_oracle, gr_oracle, yee_oracle

VARIANTS = os.path.join(GOLDEN, "variants")


def _cases():
    spec = importlib.util.spec_from_file_location(
        "make_variant_golden", os.path.join(GOLDEN, "make_variant_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return {c[0]: c for c in mod.variant_cases()}


CASES = _cases()


def test_every_case_has_a_fixture():
    have = sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(VARIANTS, "*.npz")))
    assert have == sorted(CASES), f"fixtures {have} != cases {sorted(CASES)}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference_gpu_double(name):
    _, solver, p, f64, steps = CASES[name]
    z = np.load(os.path.join(VARIANTS, name + ".npz"))
    assert str(z["solver"]) == solver and int(z["steps"]) == steps
    assert str(z["params_toml"]) == p.to_toml()
    ref = z["out_f64"]
    if solver == "sph":
        out = axisym_oracle.sph_evolve(p, np.stack([a[0] for a in f64]), steps)[:, None]
    elif solver == "cyl":
        out = axisym_oracle.cyl_evolve(p, np.stack([a[0] for a in f64]), steps)[:, None]
    elif solver == "gryee":
        out = yee_oracle.gryee_evolve(p, np.stack(f64), steps)
    elif solver == "yee":
        b0 = np.stack(f64[7:10]) if len(f64) > 7 else None
        out = yee_oracle.yee_evolve(p, np.stack(f64[:7]), steps, B0=b0)
    else:
        out = gr_oracle.gr_evolve(p, np.stack(f64), steps)
    worst = max(rel_l2(out[f], ref[f]) for f in range(7))
    assert worst < 1e-10, f"{name}: restatement vs reference double build {worst:.3e}"


def test_restatement_detects_a_planted_error():
    """The comparison is sharp: a restatement run with a perturbed parameter
    (KOeps changed by 1%) departs from the fixture far beyond the bar."""
    _, solver, p, f64, steps = CASES["sph32x16"]
    ref = np.load(os.path.join(VARIANTS, "sph32x16.npz"))["out_f64"]
    p.KOeps = p.KOeps * 1.01
    out = axisym_oracle.sph_evolve(p, np.stack([a[0] for a in f64]), steps)[:, None]
    assert max(rel_l2(out[f], ref[f]) for f in range(7)) > 1e-8


def test_staggered_restatement_keeps_div_b():
    """The staggered update's B' = c1 Bn + c2 B + c3 dB with dB = -curl E dt
    leaves the cell-centred div B unchanged up to rounding (the divergence of
    a staggered curl vanishes), also with currents, rescale and cleaning
    acting; periodic box, FP64."""
    from coffee_b200 import problems
    from oracle import yee_oracle as yo
    p = problems.alfven_params(N=12, guard=2)
    p.dt = 0.3 / 12
    rng = np.random.default_rng(2)
    shape = (16, 16, 16)
    U = np.zeros((7,) + shape)
    U[0:3] = 0.6 * rng.standard_normal((3,) + shape)
    U[3:6] = 0.5 + 0.2 * rng.standard_normal((3,) + shape)
    yo._exchange(yo.Geo(p, np.float64), list(U[:6]))
    V = yo.yee_evolve(p, U, 5)

    def div(W):
        B = W[3:6]
        c = (slice(2, 14),) * 3
        return ((np.roll(B[0], -1, 2) - B[0])[c] + (np.roll(B[1], -1, 1) - B[1])[c] +
                (np.roll(B[2], -1, 0) - B[2])[c]) * 12
    change = np.abs(div(V) - div(U)).max()
    assert change < 1e-11 * np.abs(div(U)).max()
