"""Diagnostics restated in numpy (test infrastructure: the checker of the
library's FP64 reductions, never the thing measured or shipped).

poynting_luminosity has no counterpart in the reference (which reports only
total_energy, src/algorithms/field_solver_EZ.cu:755-795); it is the
definition the library's coffee_diag_luminosity implements, written out
independently: the flux of S = E x B averaged over a shell around r,
L(r) = sum over interior points of (S . x/|x|) w(|x| - r) dx dy dz with the
tent w(s) = max(0, 1 - |s|/h) / h, h the largest grid spacing, and the EZ
point coordinate lower + delta * (i - guard) (src/data/grid.h:116-134).
"""
import numpy as np


def poynting_luminosity(p, fields, r):
    """p: SimParams-like (N, guard, lower, size); fields: 7 arrays (z, y, x)
    with guards, E then B then P.  Returns L(r) in FP64."""
    N, g = list(p.N), list(p.guard)
    d = [p.size[a] / p.N[a] for a in range(3)]
    h = max(d)
    axes = [p.lower[a] + d[a] * np.arange(N[a], dtype=np.float64) for a in range(3)]
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    R = np.sqrt(X * X + Y * Y + Z * Z)
    w = np.maximum(0.0, 1.0 - np.abs(R - r) / h) / h
    w[R <= 0] = 0.0
    sl = (slice(g[2], g[2] + N[2]), slice(g[1], g[1] + N[1]), slice(g[0], g[0] + N[0]))
    ex, ey, ez, bx, by, bz = [np.asarray(f[sl], dtype=np.float64) for f in fields[:6]]
    sx = ey * bz - ez * by
    sy = ez * bx - ex * bz
    sz = ex * by - ey * bx
    with np.errstate(invalid="ignore", divide="ignore"):
        sr = (sx * X + sy * Y + sz * Z) / R
        return float(np.nansum(sr * w) * d[0] * d[1] * d[2])
