"""Helpers shared by the tests: fixture loading and parity metrics."""
from __future__ import annotations

import glob
import os

import numpy as np

from coffee_b200.config import SimParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "P")


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = SimParams.from_toml(str(z["params_toml"]), is_text=True)
    d = {k: z[k] for k in z.files}
    return p, d


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / nb if nb > 0 else d


def interior(p):
    g = p.guard
    return tuple(slice(g[a], g[a] + p.N[a]) for a in (2, 1, 0))


# Parity bar for an FP32 result against the reference's float build.  The
# reference float build itself sits `noise` away (relative L2) from the
# same algorithm run in FP64; an independent FP32 implementation cannot be
# expected closer than that.  The bar is the larger of REL_FLOOR and
# NOISE_FACTOR * noise, per field.
REL_FLOOR = 2e-5
NOISE_FACTOR = 4.0
# ... and against the FP64 run of the same algorithm, an FP32 result must be
# no less accurate than the reference float build, up to ACC_FACTOR.
ACC_FACTOR = 2.0


def fp32_parity(out, ref32, ref64_same_algo, names=NAMES):
    """Return (ok, report) for a 7-field FP32 result."""
    ok = True
    rep = []
    for f in range(len(names)):
        noise = rel_l2(ref32[f], ref64_same_algo[f])
        vs32 = rel_l2(out[f], ref32[f])
        vs64 = rel_l2(out[f], ref64_same_algo[f])
        bar32 = max(REL_FLOOR, NOISE_FACTOR * noise)
        bar64 = ACC_FACTOR * noise + REL_FLOOR
        good = vs32 <= bar32 and vs64 <= bar64
        ok &= good
        rep.append(f"{names[f]}: vs ref32 {vs32:.2e} (bar {bar32:.1e}) vs fp64 {vs64:.2e} "
                   f"(ref32 noise {noise:.2e}, bar {bar64:.1e}){'' if good else '  <-- FAIL'}")
    return ok, "\n".join(rep)


def wide_box_case():
    """A periodic turbulence box of side 7.3 around the origin, 16^3: the
    CPU build's P-gradient taper (argument 2 (r - 3)) then spans both
    branches of its tanh, the polynomial one (|arg| <= 5/8) and the
    exponential one, and the grid is incommensurate with the modes."""
    from coffee_b200 import problems

    p = problems.turbulence_params(16)
    p.lower = [-3.65, -3.4, -3.9]
    p.size = [7.3, 7.3, 7.3]
    p.dt = 0.5 * 7.3 / 16
    return p, problems.turbulence_fields(p, np.float32)


def count_differing(a, b):
    """Number of points whose values differ (0 and -0 count as equal)."""
    return int(np.count_nonzero(np.asarray(a) != np.asarray(b)))
