"""Generate the golden fixtures of tests/golden/variants/ from the reference's
own GPU build of its log-spherical, cylindrical, GR and staggered solvers
(oracle/_ref/coffee_refgpu_double, compiled by `make -C oracle gpuref` from
the reference sources).  Needs a GPU:

    python tests/golden/make_variant_golden.py [OUTDIR [NAME ...]]

Each fixture ``<name>.npz`` holds
  params_toml  the config.toml the reference read,
  solver       "sph", "cyl", "gr", "yee" or "gryee",
  steps,
  out_f64      the double build's E (D for GR), B, P after `steps`
               evolve_fields calls, arrays of shape (d2, d1, d0).
The inputs are not stored: ``variant_cases()`` rebuilds them exactly
(float64, from coffee_b200.problems).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from coffee_b200 import problems  # noqa: E402


def variant_cases():
    """(name, solver, params, float64 input fields, steps) of every fixture."""
    out = []
    p = problems.sph_pulsar_params(nr=32, nth=16, guard=4, omega=0.25, pml=4)
    p.tp_start, p.tp_end, p.dw0, p.thp1, p.thp2 = 0.0, 0.5, 0.1, 0.6, 1.2
    out.append(("sph32x16", "sph", p, problems.sph_pulsar_fields(p, np.float64), 6))

    p = problems.sph_pulsar_params(nr=32, nth=16, guard=4, omega=0.25, pml=4)
    p.KO_geometry = False
    p.use_edotb_damping = True
    p.shift_ghost = 1
    out.append(("sph32x16_plain", "sph", p, problems.sph_pulsar_fields(p, np.float64), 6))

    p = problems.cyl_pulsar_params(nR=32, nz=64, guard=3, R_max=8.0, radius=1.5, pml=4)
    p.tp_start, p.tp_end, p.dw0, p.rpert1, p.rpert2 = 0.0, 2.0, 0.05, 3.0, 6.0
    out.append(("cyl32x64", "cyl", p, problems.cyl_pulsar_fields(p, np.float64), 6))

    p = problems.wald_params(N=16, half_size=3.0, a=0.9, pml=3)
    out.append(("gr16", "gr", p, problems.wald_fields(p, np.float64), 4))

    # staggered solver: plane Alfven wave in a periodic box, and a mixed box
    # (x periodic, absorbing layers in y and z) with a background field B0,
    # given as input arrays 7-9
    p = problems.alfven_params(N=16, guard=2)
    p.dt = 0.3 / 16
    out.append(("yee16", "yee", p, problems.alfven_plane_wave_fields(p, np.float64, yee=True), 6))
    p, f = yee_mixed_case()
    out.append(("yee_mixed16", "yee", p, f, 6))

    # staggered solver in Kerr-Schild coordinates (field_solver_gr)
    p = problems.wald_params(N=12, half_size=3.0, a=0.9, pml=2)
    out.append(("gryee12", "gryee", p, problems.wald_fields(p, np.float64, yee=True), 3))
    return out


def yee_mixed_case():
    """16 x 12 x 10 box, x periodic, weak absorbing layers in y and z, a
    non-uniform B0 and smooth perturbations with E = -v x B (|E| < |B|, so
    the reference's in-place |E| <= |B| rescale never acts): 10 arrays,
    E, B, P and then B0."""
    p = problems.alfven_params(N=16, guard=2)
    p.N = [16, 12, 10]
    p.size = [1.0, 12 / 16, 10 / 16]
    p.periodic_boundary = [True, False, False]
    p.pml = [0, 2, 2]
    p.pmllen = 2
    p.sigpml = 0.02
    p.dt = 0.25 / 16
    rng = np.random.default_rng(5)
    shape = (p.N[2] + 4, p.N[1] + 4, p.N[0] + 4)
    d = [p.size[a] / p.N[a] for a in range(3)]
    z, y, x = [(np.arange(shape[2 - a]) - 2) * d[a] for a in (2, 1, 0)]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")

    def smooth(amp):
        f = np.zeros(shape)
        for _ in range(3):
            k = rng.integers(1, 3, 3) * 2 * np.pi
            f += amp * rng.standard_normal() * np.sin(k[0] * X + k[1] * Y + k[2] * Z +
                                                      rng.uniform(0, 6.3))
        return f
    b0 = [0.8 + smooth(0.05), smooth(0.05), -0.2 + smooth(0.05)]
    B = [b0[0] + smooth(0.02), 0.2 + b0[1] + smooth(0.02), -0.1 + b0[2] + smooth(0.02)]
    v = [smooth(0.02), smooth(0.02), smooth(0.02)]
    E = [-(v[1] * B[2] - v[2] * B[1]), -(v[2] * B[0] - v[0] * B[2]),
         -(v[0] * B[1] - v[1] * B[0])]
    return p, [*E, *B, np.zeros(shape), *b0]


def main(outdir=None, only=None):
    from oracle import oracle
    outdir = outdir or os.path.join(HERE, "variants")
    os.makedirs(outdir, exist_ok=True)
    for name, solver, p, f64, steps in variant_cases():
        if only and name not in only:
            continue
        r64, _, _ = oracle.run_reference_gpu(solver, p, f64, steps)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), params_toml=p.to_toml(),
                            solver=solver, steps=steps, out_f64=np.stack(r64))
        print(name, "written")


if __name__ == "__main__":
    # make_variant_golden.py [OUTDIR [NAME ...]]: all fixtures, or the named ones
    main(sys.argv[1] if len(sys.argv) > 1 else None, sys.argv[2:] or None)
