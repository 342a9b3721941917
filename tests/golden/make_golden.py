"""Generate the golden fixtures of tests/golden/ from the reference's own
CPU build (oracle/_ref/coffee_ref_float and coffee_ref_double, compiled by
`make -C oracle ref` from the reference sources).

    python tests/golden/make_golden.py

Each fixture ``<name>.npz`` holds
  params_toml  the config.toml both builds read,
  steps, time0,
  in_f32       7 input arrays (float32; the FP64 run starts from the same
               values widened to float64),
  out_f32      the float build's E, B, P after `steps` evolve_fields calls,
  out_f64      the USE_DOUBLE build's E, B, P,
  out_f64_l16  E, B, P from the oracle restatement in FP64 with the float
               build's 16-lane P-gradient taper (field_solver_EZ.cpp:222-224
               offsets y, z by lane*delta, and the lane count differs between
               the builds), i.e. the float build's algorithm without FP32
               rounding; |out_f32 - out_f64_l16| is the FP32 noise floor,
  aux_f32      (optional) J, divE, divB of the float build's last stage.
Interior sizes are multiples of 16 because the reference CPU loop steps by
the AVX-512 width with no remainder loop (field_solver_EZ.cpp:133-137).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from coffee_b200 import problems  # noqa: E402
from oracle import oracle  # noqa: E402


def cases():
    out = []
    p = problems.alfven_params(16)
    out.append(("alfven16", p, problems.alfven_fields(p, np.float32), 5, 0.0, True))

    p = problems.turbulence_params(16)
    out.append(("turb16", p, problems.turbulence_fields(p, np.float32), 4, 0.0, False))

    p = problems.alfven_params(16)
    p.use_edotb_damping = False
    p.divB_clean = False
    p.KOeps = 0.3
    p.tau = 3.0
    out.append(("noclean16", p, problems.alfven_fields(p, np.float32), 4, 0.0, True))

    p = problems.pulsar_params(N=16, half_size=4.0, radius=1.5, omega=0.2, b0=2.0, pml=3)
    out.append(("pulsar16", p, problems.pulsar_fields(p, np.float32), 3, 0.0, True))

    p = problems.pulsar_params(N=16, half_size=4.0, radius=1.5, omega=0.2, b0=2.0, pml=3)
    p.problem = 2
    p.pert_type = 0
    p.dw0 = 0.5
    p.tp_start = 0.0
    p.tp_end = 2.0
    p.rpert1 = 1.5
    p.rpert2 = 3.0
    p.dw1 = 0.0
    out.append(("alfvenstar16", p, problems.pulsar_fields(p, np.float32), 3, 0.1, False))
    return out


def main():
    for name, p, f32, steps, t0, aux in cases():
        o32, a32, _ = oracle.run_reference(p, f32, steps, time0=t0, aux=aux)
        f64 = [a.astype(np.float64) for a in f32]
        o64, _, _ = oracle.run_reference(p, f64, steps, time0=t0, aux=False)
        o64l, _ = oracle.run_port(p, f64, steps, time0=t0, taper_lanes=16)
        kw = dict(params_toml=np.array(p.to_toml()), steps=np.array(steps), time0=np.array(t0),
                  in_f32=np.stack(f32), out_f32=np.stack(o32), out_f64=np.stack(o64),
                  out_f64_l16=np.stack(o64l))
        if aux:
            kw["aux_f32"] = np.stack(a32)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **kw)
        print(f"{name}: {os.path.getsize(path) / 1e3:.0f} kB")


if __name__ == "__main__":
    main()
