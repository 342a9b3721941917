"""numpy restatement of the reference's GR (Kerr-Schild) EZ solver.

TEST INFRASTRUCTURE ONLY: the checker for the GR kernels of coffee_b200.
Nothing in the library imports this module.

  gr_evolve  field_solver_gr_EZ::evolve_fields
             (src/algorithms/field_solver_gr_EZ.cu:858-907)
  CKS metric src/algorithms/metric_cks_impl.hpp:13-181

Arrays are (7, d2, d1, d0) = (D0, D1, D2, B0, B1, B2, P): sim_data's E holds
the electric displacement D of the 3+1 equations.  The update box is
[guard - shift, dims - guard + shift) on each axis; every kernel of the
reference that reads only its own point is applied to the whole box at once,
and the stencil kernels read slices shifted by their offsets.  Arithmetic is
in the dtype of the input (float64 for the pinned oracle).
"""
from __future__ import annotations

import math

import numpy as np

try:
    from .axisym_oracle import AS, BS, KO6, KO_CONST, as_dict, tiny
except ImportError:  # imported as a top-level module
    from axisym_oracle import AS, BS, KO6, KO_CONST, as_dict, tiny


class Cks:
    """Kerr-Schild metric functions of metric_cks_impl.hpp at (x, y, z)."""

    def __init__(self, a, x, y, z, TN):
        self.a = a
        R2 = x * x + y * y + z * z
        aa = a * a
        r = np.sqrt((R2 - aa + np.sqrt(np.maximum((R2 - aa) ** 2 + 4.0 * (a * z) ** 2, TN))) / 2.0)
        self.r = r
        r2, r3, r4 = r * r, r * r * r, r * r * r * r
        den = np.maximum(r4 + aa * z * z, TN)                    # r^4 + a^2 z^2
        denu = np.maximum(2.0 * r3 + r4 + aa * z * z, TN)        # 2 r^3 + r^4 + a^2 z^2
        ar = np.maximum(aa + r2, TN)
        ar2 = np.maximum((aa + r2) ** 2, TN)
        lx, ly = r * x + a * y, -a * x + r * y
        self.gamma = 1.0 + 2.0 * r3 / den
        self.sqrt_gamma = np.sqrt(self.gamma)
        self.alpha = np.sqrt(1.0 / (1.0 + 2.0 * r3 / den))
        self.beta_u = (2.0 * r3 * lx / ar / denu, 2.0 * r3 * ly / ar / denu, 2.0 * r2 * z / denu)
        self.gd = {
            11: 1.0 + 2.0 * r3 * lx * lx / ar2 / den,
            12: 2.0 * r3 * lx * ly / ar2 / den,
            13: 2.0 * r2 * lx * z / ar / den,
            22: 1.0 + 2.0 * r3 * (a * x - r * y) ** 2 / ar2 / den,
            23: 2.0 * r2 * ly * z / ar / den,
            33: 1.0 + 2.0 * r * z * z / den,
        }
        self.gu = {
            11: 1.0 - 2.0 * r3 * lx * lx / ar2 / denu,
            12: -2.0 * r3 * lx * ly / ar2 / denu,
            13: -2.0 * r2 * lx * z / ar / denu,
            22: 1.0 - 2.0 * r3 * (a * x - r * y) ** 2 / ar2 / denu,
            23: 2.0 * r2 * (a * x - r * y) * z / ar / denu,
            33: 1.0 - 2.0 * r * z * z / denu,
        }

    def lower(self, v):
        g = self.gd
        return (g[11] * v[0] + g[12] * v[1] + g[13] * v[2],
                g[12] * v[0] + g[22] * v[1] + g[23] * v[2],
                g[13] * v[0] + g[23] * v[1] + g[33] * v[2])

    def raise_(self, v):
        g = self.gu
        return (g[11] * v[0] + g[12] * v[1] + g[13] * v[2],
                g[12] * v[0] + g[22] * v[1] + g[23] * v[2],
                g[13] * v[0] + g[23] * v[1] + g[33] * v[2])


def gr_evolve(p, U: np.ndarray, nsteps: int, time0: float = 0.0, want_aux: bool = False):
    """Advance U (7, d2, d1, d0) by nsteps evolve_fields calls of the
    reference's GR EZ solver.  Returns U (and aux = J, divD, divB of the last
    stage when want_aux)."""
    p = as_dict(p)
    T = U.dtype.type
    U = U.copy()
    TN = tiny(T)
    N, g, s = p["N"], p["guard"], p["shift_ghost"]
    dims = [N[a] + 2 * g[a] for a in range(3)]
    delta = [T(p["size"][a]) / T(N[a]) for a in range(3)]
    inv = [T(1.0) / d for d in delta]
    lo = [g[a] - s for a in range(3)]
    hi = [dims[a] - g[a] + s for a in range(3)]
    a = T(p["a"])
    dt = T(p["dt"])
    coords = [T(p["lower"][ax]) + delta[ax] * (np.arange(dims[ax]) - g[ax]).astype(T)
              for ax in range(3)]
    Zf, Yf, Xf = np.meshgrid(coords[2], coords[1], coords[0], indexing="ij")
    full = Cks(a, Xf, Yf, Zf, TN)

    def bx(f, dk=0, dj=0, di=0):
        return f[lo[2] + dk:hi[2] + dk, lo[1] + dj:hi[1] + dj, lo[0] + di:hi[0] + di]

    Xb, Yb, Zb = bx(Xf), bx(Yf), bx(Zf)
    m = Cks(a, Xb, Yb, Zb, TN)
    offs = {0: (0, 0, 1), 1: (0, 1, 0), 2: (1, 0, 0)}

    def sh(f, ax, k):
        dk, dj, di = (k * o for o in offs[ax])
        return bx(f, dk, dj, di)

    def d1(f, ax):
        """df1 = diff1_4 * inv_delta (finite_diff.h:14-19, 79-82)."""
        return (sh(f, ax, -2) - 8.0 * sh(f, ax, -1) + 8.0 * sh(f, ax, 1)
                - sh(f, ax, 2)) / 12.0 * inv[ax]

    def sg_at(ax, k):
        """sqrt(gamma) at the box points shifted by k * delta along ax."""
        d = [0.0, 0.0, 0.0]
        d[ax] = k * delta[ax]
        return Cks(a, Xb + d[0], Yb + d[1], Zb + d[2], TN).sqrt_gamma

    sg_cache = {(ax, k): sg_at(ax, k) for ax in range(3) for k in (-2, -1, 1, 2)}

    def div4(f):
        """div4 (field_solver_gr_EZ.cu:44-86)."""
        tot = 0.0
        for ax in range(3):
            tot = tot + (sh(f[ax], ax, -2) * sg_cache[(ax, -2)]
                         - 8.0 * sh(f[ax], ax, -1) * sg_cache[(ax, -1)]
                         + 8.0 * sh(f[ax], ax, 1) * sg_cache[(ax, 1)]
                         - sh(f[ax], ax, 2) * sg_cache[(ax, 2)]) / 12.0 / delta[ax]
        return tot / m.sqrt_gamma

    dU = np.zeros_like(U)
    aux = np.zeros((5,) + U.shape[1:], T)
    r0, dl = 5.0, 1.0
    shape = 0.5 * (1.0 - np.tanh((m.r - r0) / dl))  # (:276-278)

    def compute_EH():
        """kernel_compute_E_gr / kernel_compute_H_gr (:88-186), full grid."""
        D, B = U[0:3], U[3:6]
        Dd, Bd = full.lower(D), full.lower(B)
        bu, al, sgm = full.beta_u, full.alpha, full.sqrt_gamma
        E = (al * Dd[0] + sgm * (bu[1] * B[2] - bu[2] * B[1]),
             al * Dd[1] + sgm * (bu[2] * B[0] - bu[0] * B[2]),
             al * Dd[2] + sgm * (bu[0] * B[1] - bu[1] * B[0]))
        H = (al * Bd[0] - sgm * (bu[1] * D[2] - bu[2] * D[1]),
             al * Bd[1] - sgm * (bu[2] * D[0] - bu[0] * D[2]),
             al * Bd[2] - sgm * (bu[0] * D[1] - bu[1] * D[0]))
        return E, H

    def curl(F):
        gms = m.sqrt_gamma
        return ((d1(F[2], 1) - d1(F[1], 2)) / gms,
                (d1(F[0], 2) - d1(F[2], 0)) / gms,
                (d1(F[1], 0) - d1(F[0], 1)) / gms)

    def rk_stage(As, Bs):
        """kernel_rk_step1_gr + kernel_rk_step2_gr (:188-420)."""
        E, H = compute_EH()
        rotH, rotE = curl(H), curl(E)
        D, B, P = U[0:3], U[3:6], U[6]
        divD, divB = div4(D), div4(B)
        b = [bx(c) for c in B]
        d = [bx(c) for c in D]
        e = [bx(c) for c in E]
        Bd, Dd = m.lower(b), m.lower(d)
        gms = m.sqrt_gamma
        if p["calc_current"]:
            B2 = np.maximum(b[0] * Bd[0] + b[1] * Bd[1] + b[2] * Bd[2], TN)
            Jp = (Bd[0] * rotH[0] + Bd[1] * rotH[1] + Bd[2] * rotH[2]) - \
                 (Dd[0] * rotE[0] + Dd[1] * rotE[1] + Dd[2] * rotE[2])
            J = ((divD * (e[1] * Bd[2] - e[2] * Bd[1]) / gms + Jp * b[0]) / B2,
                 (divD * (e[2] * Bd[0] - e[0] * Bd[2]) / gms + Jp * b[1]) / B2,
                 (divD * (e[0] * Bd[1] - e[1] * Bd[0]) / gms + Jp * b[2]) / B2)
        else:
            J = (0.0, 0.0, 0.0)
        Pd = (d1(P, 0), d1(P, 1), d1(P, 2))
        Pu = m.raise_(Pd)
        al, bu = m.alpha, m.beta_u
        for c in range(3):
            if p["divB_clean"]:
                rhsB = dt * (-rotE[c] + (-al * Pu[c] + bu[c] * divB) * shape)
            else:
                rhsB = -dt * rotE[c]
            bx(dU[3 + c])[...] = As * bx(dU[3 + c]) + rhsB
            bx(dU[c])[...] = As * bx(dU[c]) + dt * (rotH[c] - J[c])
        bx(dU[6])[...] = As * bx(dU[6]) + dt * (-al * divB + bu[0] * Pd[0] + bu[1] * Pd[1]
                                                + bu[2] * Pd[2]) - al * bx(P) / p["tau"]
        for c in range(3):
            bx(aux[c])[...] = J[c]
        bx(aux[3])[...] = divD
        bx(aux[4])[...] = divB
        for f in range(7):
            bx(U[f])[...] = bx(U[f]) + Bs * bx(dU[f])

    def clean_epar():
        """kernel_clean_epar_gr (:422-463)."""
        d = [bx(U[c]) for c in range(3)]
        b = [bx(U[3 + c]) for c in range(3)]
        Bd = m.lower(b)
        B2 = np.maximum(b[0] * Bd[0] + b[1] * Bd[1] + b[2] * Bd[2], TN)
        DB = d[0] * Bd[0] + d[1] * Bd[1] + d[2] * Bd[2]
        for c in range(3):
            d[c][...] = d[c] - DB * b[c] / B2

    def check_egb():
        """kernel_check_eGTb_gr (:465-521)."""
        d = [bx(U[c]) for c in range(3)]
        b = [bx(U[3 + c]) for c in range(3)]
        Dd, Bd = m.lower(d), m.lower(b)
        D2 = np.maximum(d[0] * Dd[0] + d[1] * Dd[1] + d[2] * Dd[2], TN)
        B2 = b[0] * Bd[0] + b[1] * Bd[1] + b[2] * Bd[2]
        with np.errstate(invalid="ignore"):
            tmp = np.where(D2 > B2, np.sqrt(B2 / D2), 1.0)
        for c in range(3):
            d[c][...] = tmp * d[c]

    def absorbing(Un):
        """kernel_boundary_absorbing_thread (boundary.cu:17-79) and
        kernel_absorbing_inner (field_solver_gr_EZ.cu:610-701)."""
        sig = 0.0
        pos = (Xb, Yb, Zb)
        out = np.zeros_like(Xb, dtype=bool)
        for ax in range(3):
            xh = p["lower"][ax] + p["size"][ax] - p["pml"][ax] * delta[ax]
            xl = p["lower"][ax] + p["pml"][ax] * delta[ax]
            out |= (pos[ax] > xh) | (pos[ax] < xl)
            scale = p["pmllen"] * delta[0]
            x = pos[ax]
            sig = sig + np.where(x > xh, p["sigpml"] * ((x - xh) / scale) ** 3,
                                 np.where(x < xl, p["sigpml"] * ((xl - x) / scale) ** 3, 0.0))
        on = out & (sig > TN)
        with np.errstate(invalid="ignore", divide="ignore"):
            ex = np.exp(-sig)
            fac = np.where(on, (1.0 - ex) / np.where(on, sig, 1.0), 0.0)
        for c in range(6):
            u, un = bx(U[c]), bx(Un[c])
            u[...] = np.where(on, ex * un + fac * (u - un), u)
        rH = 1.0 + math.sqrt(1.0 - float(a) ** 2)
        r1, r2, dd = 0.7 * rH, 0.01 * rH, 0.2 * rH
        r = m.r
        sig = p["sigpml"] * ((r1 - r) / dd) ** 3 * dt
        on = (r < r1) & (sig > TN)
        with np.errstate(invalid="ignore", divide="ignore"):
            ex = np.exp(-sig)
            fac = np.where(on, (1.0 - ex) / np.where(on, sig, 1.0), 0.0)
        for c in range(6):
            u, un = bx(U[c]), bx(Un[c])
            u[...] = np.where(on, ex * un + fac * (u - un), u)
            u[...] = np.where(r < r2, 0.0, u)

    def ko():
        """kernel_KO_step1_gr / _step2_gr (:523-608); KO of finite_diff.h:84-92."""
        tmp = []
        for f in range(7):
            t = 0.0
            for ax in range(3):
                t = t + sum(c * sh(U[f], ax, k) for c, k in zip(KO6, range(-3, 4)))
            tmp.append(t)
        for f in range(7):
            bx(U[f])[...] = bx(U[f]) - p["KOeps"] * KO_CONST * tmp[f]

    def periodic():
        for ax in range(3):
            if not p["periodic_boundary"][ax]:
                continue
            gg, n = g[ax], dims[ax] - 2 * g[ax]
            idx = [slice(None)] * 4
            src = list(idx)
            idx[3 - ax] = slice(n + gg, n + 2 * gg)
            src[3 - ax] = slice(gg, 2 * gg)
            U[tuple(idx)] = U[tuple(src)]
            idx[3 - ax] = slice(0, gg)
            src[3 - ax] = slice(n, n + gg)
            U[tuple(idx)] = U[tuple(src)]

    for _ in range(nsteps):
        Un = U.copy()
        for st in range(5):
            rk_stage(T(AS[st]), T(BS[st]))
            if p["clean_ep"]:
                clean_epar()
            if p["check_egb"]:
                check_egb()
            if st == 4:
                absorbing(Un)
            periodic()
        ko()
        if p["clean_ep"]:
            clean_epar()
        if p["check_egb"]:
            check_egb()
        periodic()
    return (U, aux) if want_aux else U
