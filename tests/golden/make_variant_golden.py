"""Generate the golden fixtures of tests/golden/variants/ from the reference's
own GPU build of its log-spherical, cylindrical and GR solvers
(oracle/_ref/coffee_refgpu_double, compiled by `make -C oracle gpuref` from
the reference sources).  Needs a GPU:

    python tests/golden/make_variant_golden.py [OUTDIR]

Each fixture ``<name>.npz`` holds
  params_toml  the config.toml the reference read,
  solver       "sph", "cyl" or "gr",
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
    return out


def main(outdir=None):
    from oracle import oracle
    outdir = outdir or os.path.join(HERE, "variants")
    os.makedirs(outdir, exist_ok=True)
    for name, solver, p, f64, steps in variant_cases():
        r64, _, _ = oracle.run_reference_gpu(solver, p, f64, steps)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), params_toml=p.to_toml(),
                            solver=solver, steps=steps, out_f64=np.stack(r64))
        print(name, "written")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
