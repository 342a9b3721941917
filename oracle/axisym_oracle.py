"""numpy restatement of the reference's two 2D axisymmetric GPU EZ solvers.

TEST INFRASTRUCTURE ONLY: the checker for the log-spherical and cylindrical
kernels of coffee_b200.  Nothing in the library imports this module.

  sph_evolve  field_solver_EZ_spherical::evolve_fields
              (src/algorithms/field_solver_EZ_spherical.cu:958-1012)
  cyl_evolve  field_solver_EZ_cylindrical::evolve_fields
              (src/algorithms/field_solver_EZ_cylindrical.cu:674-713)

Both run on one z plane: arrays are (7, d1, d0) = (E0, E1, E2, B0, B1, B2, P)
with guard cells, index [component, j, i] (the reference layout i + j*d0).
Every kernel of the reference touches the update box
[guard - shift, dims - guard + shift) of axes 0 and 1; the box is handled as
one numpy slice per stencil offset, and a kernel that reads only its own point
is applied to the whole box at once, which is what the reference computes as
the kernels write nothing their own box reads.

The arithmetic is carried out in the dtype of the input (float64 for the
pinned oracle).  Reference quirks are kept: the P damping term -P/tau is not
multiplied by dt (spherical.cu:319-320, cylindrical.cu:197-198); the
cylindrical solver keeps its own P (field_solver_EZ_cylindrical.h:10) and
uses stage times shifted by one (cylindrical.cu:684-685); the spherical
Pz = 0 / gamma_33 is NaN on the theta = 0 row, as in the reference, and that
row is then reset by the axis boundary.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass

import numpy as np

# LSRK(5,4) coefficients, src/algorithms/field_solver_EZ_spherical.cu:960-965
AS = (0.0, -0.4178904745, -1.192151694643, -1.697784692471, -1.514183444257)
BS = (0.1496590219993, 0.3792103129999, 0.8229550293869, 0.6994504559488,
      0.1530572479681)
CS_SPH = (0.0, 0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306784)
# field_solver_EZ_cylindrical.cu:684-685
CS_CYL = (0.1496590219993, 0.3704009573644, 0.6222557631345, 0.9582821306784, 1.0)
KO_CONST = -1.0 / 64.0  # 6th-order dissipation (spherical.cu:505-513)
KO6 = (1.0, -6.0, 15.0, -20.0, 15.0, -6.0, 1.0)


def tiny(dtype) -> float:
    """TINY of src/data/typedefs.h:6-12."""
    return 1e-7 if np.dtype(dtype) == np.float32 else 1e-11


@dataclass
class Plane:
    """Grid of one 2D run: dims/guard/lower/delta of axes 0 and 1, the update
    box and the periodic flags (src/data/grid.h:116-134; pos(n) with stagger
    bit 1 is lower + delta * (n - guard))."""
    d0: int
    d1: int
    g0: int
    g1: int
    lower: tuple
    delta: tuple
    shift: int
    periodic: tuple

    @property
    def box(self):
        s = self.shift
        return (self.g1 - s, self.d1 - self.g1 + s, self.g0 - s, self.d0 - self.g0 + s)


def as_dict(p) -> dict:
    """Parameters as a dict (accepts coffee_b200.config.SimParams)."""
    return p if isinstance(p, dict) else dataclasses.asdict(p)


def plane_from_params(p) -> Plane:
    p = as_dict(p)
    N, g = p["N"], p["guard"]
    size, lower = p["size"], p["lower"]
    return Plane(N[0] + 2 * g[0], N[1] + 2 * g[1], g[0], g[1],
                 (lower[0], lower[1]), (size[0] / N[0], size[1] / N[1]),
                 p.get("shift_ghost", 0), tuple(p.get("periodic_boundary", (0, 0, 0))[:2]))


class _Box:
    """Slices of the update box shifted by (dj, di)."""

    def __init__(self, pl: Plane):
        self.j0, self.j1, self.i0, self.i1 = pl.box

    def __call__(self, f, dj=0, di=0):
        return f[self.j0 + dj:self.j1 + dj, self.i0 + di:self.i1 + di]


def _periodic_fill(U, pl: Plane):
    """Single-rank guard exchange of the periodic axes, x then y
    (src/sim_env_impl.hpp:180-195 with both neighbours = self)."""
    if pl.periodic[0]:
        g, n = pl.g0, pl.d0 - 2 * pl.g0
        U[..., :, n + g:n + 2 * g] = U[..., :, g:2 * g]
        U[..., :, 0:g] = U[..., :, n:n + g]
    if pl.periodic[1]:
        g, n = pl.g1, pl.d1 - 2 * pl.g1
        U[..., n + g:n + 2 * g, :] = U[..., g:2 * g, :]
        U[..., 0:g, :] = U[..., n:n + g, :]


def _d1(f, bx, axis, inv):
    """diff1_4 * inv_delta (src/algorithms/finite_diff.h:14-19, 79-82)."""
    if axis == 0:
        return (bx(f, 0, -2) - 8.0 * bx(f, 0, -1) + 8.0 * bx(f, 0, 1) - bx(f, 0, 2)) / 12.0 * inv
    return (bx(f, -2, 0) - 8.0 * bx(f, -1, 0) + 8.0 * bx(f, 1, 0) - bx(f, 2, 0)) / 12.0 * inv


def _d6(f, bx, axis):
    """diff6_2 (src/algorithms/finite_diff.h:27-31)."""
    out = 0.0
    for c, k in zip(KO6, range(-3, 4)):
        out = out + c * (bx(f, 0, k) if axis == 0 else bx(f, k, 0))
    return out


# ---------------------------------------------------------------------------
# log-spherical (x = ln r, y = theta), src/algorithms/metric_sph.h:90-133
# ---------------------------------------------------------------------------
def _sph_metric(x, y):
    r = np.exp(x)
    g11 = r * r
    g22 = r * r
    g33 = np.square(r * np.sin(y))
    return r, g11, g22, g33


def _sph_sqrt_gamma(x, y):
    _, g11, g22, g33 = _sph_metric(x, y)
    return np.sqrt(g11 * g22 * g33)


def _wpert_sph_angle(t, th, tp_start, tp_end, dw0, nT, thp1, thp2):
    """wpert_sph_angle (field_solver_EZ_spherical.cu:576-595)."""
    if thp1 > thp2:
        thp1, thp2 = thp2, thp1
    mu = (thp1 + thp2) / 2.0
    if not (tp_start <= t <= tp_end):
        return np.zeros_like(th)
    val = (dw0 * np.square(np.cos((th - mu) * math.pi / (thp2 - thp1)))
           * math.sin((t - tp_start) * math.pi / (tp_end - tp_start)) ** 2
           * math.sin((t - tp_start) * 2.0 * math.pi * nT / (tp_end - tp_start)))
    return np.where((th >= thp1) & (th <= thp2), val, 0.0)


def sph_evolve(p, U: np.ndarray, nsteps: int, time0: float = 0.0, want_aux: bool = False):
    """Advance U (7, d1, d0) by nsteps evolve_fields calls of the reference's
    log-spherical solver; returns U, or (U, aux) with aux = (J0, J1, J2,
    divE, divB) of the last stage (written to B0/divE/divB by
    kernel_rk_step1_sph, field_solver_EZ_spherical.cu:322-327)."""
    p = as_dict(p)
    T = U.dtype.type
    U = U.reshape(7, U.shape[-2], U.shape[-1]).copy()
    pl = plane_from_params(p)
    bx = _Box(pl)
    TN = tiny(T)
    dU = np.zeros((7, pl.d1, pl.d0), T)
    aux = np.zeros((5, pl.d1, pl.d0), T)
    dt = T(p["dt"])
    x = (T(pl.lower[0]) + T(pl.delta[0]) * (np.arange(pl.d0) - pl.g0).astype(T)).astype(T)
    y = (T(pl.lower[1]) + T(pl.delta[1]) * (np.arange(pl.d1) - pl.g1).astype(T)).astype(T)
    X, Y = np.meshgrid(x, y)
    r, g11, g22, g33 = _sph_metric(X, Y)
    dx, dy = T(pl.delta[0]), T(pl.delta[1])
    inv0, inv1 = T(1.0) / dx, T(1.0) / dy
    Xb, Yb = bx(X), bx(Y)
    sg = lambda ox, oy: _sph_sqrt_gamma(Xb + ox * dx, Yb + oy * dy)  # noqa: E731
    gms = np.maximum(bx(_sph_sqrt_gamma(X, Y)), TN)
    g11b, g22b, g33b, rb = bx(g11), bx(g22), bx(g33), bx(r)
    radius, b0, omega = p["radius"], p["b0"], p["omega"]

    def div4(fx, fy):
        """div4_sph (field_solver_EZ_spherical.cu:99-124)."""
        tx = (bx(fx, 0, -2) * sg(-2, 0) - 8.0 * bx(fx, 0, -1) * sg(-1, 0)
              + 8.0 * bx(fx, 0, 1) * sg(1, 0) - bx(fx, 0, 2) * sg(2, 0)) / 12.0 * inv0
        ty = (bx(fy, -2, 0) * sg(0, -2) - 8.0 * bx(fy, -1, 0) * sg(0, -1)
              + 8.0 * bx(fy, 1, 0) * sg(0, 1) - bx(fy, 2, 0) * sg(0, 2)) / 12.0 * inv1
        return (tx + ty + 0.0) / gms

    def rk_stage(As, Bs):
        """kernel_compute_ElBl + kernel_rk_step1_sph + kernel_rk_step2_sph
        (field_solver_EZ_spherical.cu:175-359)."""
        E, B, P = U[0:3], U[3:6], U[6]
        El = (g11 * E[0], g22 * E[1], g33 * E[2])
        Bl = (g11 * B[0], g22 * B[1], g33 * B[2])
        rotBx = (_d1(Bl[2], bx, 1, inv1) - 0.0) / gms
        rotEx = (_d1(El[2], bx, 1, inv1) - 0.0) / gms
        rotBy = (0.0 - _d1(Bl[2], bx, 0, inv0)) / gms
        rotBz = (_d1(Bl[1], bx, 0, inv0) - _d1(Bl[0], bx, 1, inv1)) / gms
        rotEy = (0.0 - _d1(El[2], bx, 0, inv0)) / gms
        rotEz = (_d1(El[1], bx, 0, inv0) - _d1(El[0], bx, 1, inv1)) / gms
        divE = div4(E[0], E[1])
        divB = div4(B[0], B[1])
        e = [bx(c) for c in E]
        b = [bx(c) for c in B]
        el = [bx(c) for c in El]
        bl = [bx(c) for c in Bl]
        B2 = np.maximum(b[0] * bl[0] + b[1] * bl[1] + b[2] * bl[2], TN)
        if p["calc_current"]:
            Jp = (bl[0] * rotBx + bl[1] * rotBy + bl[2] * rotBz) - \
                 (el[0] * rotEx + el[1] * rotEy + el[2] * rotEz)
            cx = el[1] * bl[2] - el[2] * bl[1]
            cy = el[2] * bl[0] - el[0] * bl[2]
            cz = el[0] * bl[1] - el[1] * bl[0]
            if p["use_edotb_damping"]:
                E2 = e[0] * el[0] + e[1] * el[1] + e[2] * el[2]
                chi2 = B2 - E2
                EdotB = e[0] * bl[0] + e[1] * bl[1] + e[2] * bl[2]
                E02 = 0.5 * (np.sqrt(chi2 * chi2 + 4.0 * EdotB * EdotB) - chi2)
                Jp = Jp + p["damp_gamma"] * EdotB / dt
                J = [divE * c / gms / (E02 + B2) + Jp * bb / B2
                     for c, bb in zip((cx, cy, cz), b)]
            else:
                J = [(divE * c / gms + Jp * bb) / B2 for c, bb in zip((cx, cy, cz), b)]
        else:
            J = [np.zeros_like(B2)] * 3
        if p["divB_clean"]:
            with np.errstate(invalid="ignore", divide="ignore"):
                Pg = (_d1(P, bx, 0, inv0) / g11b, _d1(P, bx, 1, inv1) / g22b, 0.0 / g33b)
        else:
            Pg = (0.0, 0.0, 0.0)
        rotE, rotB = (rotEx, rotEy, rotEz), (rotBx, rotBy, rotBz)
        with np.errstate(invalid="ignore"):
            for c in range(3):
                bx(dU[3 + c])[...] = As * bx(dU[3 + c]) - dt * (rotE[c] + Pg[c])
                bx(dU[c])[...] = As * bx(dU[c]) + dt * (rotB[c] - J[c])
            bx(dU[6])[...] = As * bx(dU[6]) - dt * p["ch2"] * divB - bx(P) / p["tau"]
            for c in range(3):
                bx(aux[c])[...] = J[c]
            bx(aux[3])[...] = divE
            bx(aux[4])[...] = divB
            for f in range(7):
                bx(U[f])[...] = bx(U[f]) + Bs * bx(dU[f])

    def metric_sq(V):
        return g11b * V[0] * V[0] + g22b * V[1] * V[1] + g33b * V[2] * V[2]

    def clean_epar():
        """kernel_Epar_sph (field_solver_EZ_spherical.cu:361-399)."""
        E = [bx(U[c]) for c in range(3)]
        B = [bx(U[3 + c]) for c in range(3)]
        with np.errstate(invalid="ignore"):
            B2 = metric_sq(B)
            B2 = np.where(B2 < TN, TN, B2)
            EB = g11b * E[0] * B[0] + g22b * E[1] * B[1] + g33b * E[2] * B[2]
            for c in range(3):
                E[c][...] = E[c] - EB / B2 * B[c]

    def check_egb():
        """kernel_EgtB_sph (field_solver_EZ_spherical.cu:401-442)."""
        E = [bx(U[c]) for c in range(3)]
        B = [bx(U[3 + c]) for c in range(3)]
        with np.errstate(invalid="ignore", divide="ignore"):
            B2 = metric_sq(B)
            B2 = np.where(B2 < TN, TN, B2)
            E2 = metric_sq(E)
            s = np.where(E2 > B2, np.sqrt(B2 / E2), 1.0)
            for c in range(3):
                E[c][...] = np.where(E2 > B2, E[c] * s, E[c])

    def boundary_pulsar(t):
        """kernel_boundary_pulsar_sph (field_solver_EZ_spherical.cu:617-688)."""
        th = Yb
        w = omega + _wpert_sph_angle(t, th, p["tp_start"], p["tp_end"], p["dw0"], p["nT"],
                                     p["thp1"], p["thp2"]) \
            + _wpert_sph_angle(t, th, p["tp_start1"], p["tp_end1"], p["dw1"], p["nT1"],
                               p["thp11"], p["thp21"])
        inner = rb < radius + dx
        bxn = b0 * (2.0 * np.cos(th) / rb ** 3)
        byn = b0 * (np.sin(th) / rb ** 3)
        v3n = w * rb * np.sin(th)
        exn = v3n * byn
        eyn = -v3n * bxn
        g11s, g22s = np.sqrt(g11b), np.sqrt(g22b)
        surf = inner & (np.abs(rb - radius) < dx / 2.0)
        core = inner & ~surf & (rb < radius - TN)
        Ex, Ey, Ez, Bx_, By_, Bz_ = (bx(U[c]) for c in range(6))
        Bx_[surf] = (bxn / g11s)[surf]
        Ey[surf] = (eyn / g22s)[surf]
        Ez[surf] = 0.0
        Bx_[core] = (bxn / g11s)[core]
        By_[core] = (byn / g22s)[core]
        Bz_[core] = 0.0
        Ex[core] = (exn / g11s)[core]
        Ey[core] = (eyn / g22s)[core]
        Ez[core] = 0.0

    def boundary_axis():
        """kernel_boundary_axis_sph (field_solver_EZ_spherical.cu:690-748)."""
        i0, i1 = bx.i0, bx.i1
        j = pl.g1
        if abs(y[j]) < dy / 2.0:
            for c, keep in ((0, 1), (1, 0), (2, 0), (3, 1), (4, 0), (5, 0)):
                U[c, j, i0:i1] = U[c, j + 1, i0:i1] if keep else 0.0
            U[6, j, i0:i1] = U[6, j + 1, i0:i1]
            for l in range(1, 4):
                for c, sgn in ((0, 1), (1, -1), (2, -1), (3, 1), (4, -1), (5, -1)):
                    U[c, j - l, i0:i1] = sgn * U[c, j + l, i0:i1]
        j = pl.d1 - pl.g1
        if abs(y[j] - math.pi) < dy / 2.0:
            for c, keep in ((0, 1), (1, 0), (2, 0), (3, 1), (4, 0), (5, 0)):
                U[c, j, i0:i1] = U[c, j - 1, i0:i1] if keep else 0.0
            U[6, j, i0:i1] = U[6, j - 1, i0:i1]
            for l in range(1, 4):
                for c, sgn in ((0, 1), (1, -1), (2, -1), (3, 1), (4, -1), (5, -1)):
                    U[c, j + l, i0:i1] = sgn * U[c, j - l, i0:i1]

    def boundary_absorbing(Un):
        """kernel_boundary_absorbing_sph (field_solver_EZ_spherical.cu:758-802)."""
        xh = p["lower"][0] + p["size"][0] - p["pml"][0] * dx
        rh = math.exp(xh)
        with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
            sig = np.where(rb > rh, p["sigpml"] * ((rb - rh) / (p["pmllen"] * 1.0)) ** 3, 0.0)
            on = (Xb > xh) & (sig > TN)
            ex = np.exp(-sig)
            fac = np.where(on, (1.0 - ex) / np.where(on, sig, 1.0), 0.0)
            for c in range(6):
                u, un = bx(U[c]), bx(Un[c])
                u[...] = np.where(on, ex * un + fac * (u - un), u)

    def ko():
        """kernel_KO_step1_sph / _step2_sph (field_solver_EZ_spherical.cu:444-555)."""
        tmp = []
        for f in range(7):
            F = U[f]
            if p["KO_geometry"]:
                tx = sum(c * bx(F, 0, k) * sg(k, 0) for c, k in zip(KO6, range(-3, 4)))
                ty = sum(c * bx(F, k, 0) * sg(0, k) for c, k in zip(KO6, range(-3, 4)))
                tmp.append((tx + ty) / gms)
            else:
                tmp.append(_d6(F, bx, 0) + _d6(F, bx, 1))
        for f in range(7):
            bx(U[f])[...] = bx(U[f]) - p["KOeps"] * KO_CONST * tmp[f]

    time = T(time0)
    for _ in range(nsteps):
        boundary_axis()
        Un = U.copy()
        for s in range(5):
            rk_stage(T(AS[s]), T(BS[s]))
            if p["clean_ep"]:
                clean_epar()
            if p["check_egb"]:
                check_egb()
            boundary_pulsar(time + T(CS_SPH[s]) * dt)
            if s == 4:
                boundary_absorbing(Un)
            boundary_axis()
            _periodic_fill(U, pl)
        ko()
        if p["clean_ep"]:
            clean_epar()
        if p["check_egb"]:
            check_egb()
        boundary_pulsar(time + dt)
        boundary_axis()
        _periodic_fill(U, pl)
        time = T(time + dt)
    return (U, aux) if want_aux else U


# ---------------------------------------------------------------------------
# cylindrical (x = R, y = z), src/algorithms/field_solver_EZ_cylindrical.cu
# components 0 E_R, 1 E_z, 2 E_phi, 3 B_R, 4 B_z, 5 B_phi
# ---------------------------------------------------------------------------
def _pmlsigma(x, xl, xh, scale, sig0):
    """pmlsigma (src/algorithms/boundary.cu:7-15)."""
    return np.where(x > xh, sig0 * ((x - xh) / scale) ** 3,
                    np.where(x < xl, sig0 * ((xl - x) / scale) ** 3, 0.0))


def cyl_evolve(p, U: np.ndarray, nsteps: int, time0: float = 0.0):
    """Advance U (7, d1, d0) by nsteps evolve_fields calls of the reference's
    cylindrical solver (field_solver_EZ_cylindrical.cu:674-713).  P is the
    solver's own P (loaded from U[6])."""
    p = as_dict(p)
    T = U.dtype.type
    U = U.reshape(7, U.shape[-2], U.shape[-1]).copy()
    pl = plane_from_params(p)
    bx = _Box(pl)
    TN = tiny(T)
    dt = T(p["dt"])
    dR, dz = T(pl.delta[0]), T(pl.delta[1])
    Rv = (T(pl.lower[0]) + dR * (np.arange(pl.d0) - pl.g0).astype(T)).astype(T)
    zv = (T(pl.lower[1]) + dz * (np.arange(pl.d1) - pl.g1).astype(T)).astype(T)
    Zg, Rg = np.meshgrid(zv, Rv, indexing="ij")
    Rb, Zb = bx(Rg), bx(Zg)
    Rc = np.where(np.abs(Rb) < TN, TN, Rb)  # kernel_rk_step1_thread (:165-167)
    dU = np.zeros((7, pl.d1, pl.d0), T)
    radius, b0 = p["radius"], p["b0"]

    def dfdR(f):
        return (bx(f, 0, -2) - 8 * bx(f, 0, -1) + 8 * bx(f, 0, 1) - bx(f, 0, 2)) / 12.0 / dR

    def dfdz(f):
        return (bx(f, -2, 0) - 8 * bx(f, -1, 0) + 8 * bx(f, 1, 0) - bx(f, 2, 0)) / 12.0 / dz

    def dfRdRR(f):
        """(:110-113): 2 f_R on the axis, else (R f)_R / R."""
        h = dR
        rr = (bx(f, 0, -2) * (Rc - 2 * h) - 8 * bx(f, 0, -1) * (Rc - h)
              + 8 * bx(f, 0, 1) * (Rc + h) - bx(f, 0, 2) * (Rc + 2 * h)) / 12.0 / dR / Rc
        return np.where(np.abs(Rc) < dR / 4.0, 2.0 * dfdR(f), rr)

    def rk_stage(As, Bs):
        """kernel_rk_step1_thread + kernel_rk_step2_thread (:143-234)."""
        ER, Ez, Ef, BR, Bz, Bf, P = U
        rotBR, rotBz, rotBf = -dfdz(Bf), dfRdRR(Bf), dfdz(BR) - dfdR(Bz)
        rotER, rotEz, rotEf = -dfdz(Ef), dfRdRR(Ef), dfdz(ER) - dfdR(Ez)
        divE = dfRdRR(ER) + dfdz(Ez)
        divB = dfRdRR(BR) + dfdz(Bz)
        er, ez, ef, br, bz, bf, pp = (bx(c) for c in U)
        B2 = np.maximum(br * br + bz * bz + bf * bf, TN)
        Jp = (br * rotBR + bz * rotBz + bf * rotBf) - (er * rotER + ez * rotEz + ef * rotEf)
        JR = (divE * (ef * bz - ez * bf) + Jp * br) / B2
        Jf = (divE * (ez * br - er * bz) + Jp * bf) / B2
        Jz = (divE * (er * bf - ef * br) + Jp * bz) / B2
        rhs = (dt * (rotBR - JR), dt * (rotBz - Jz), dt * (rotBf - Jf),
               -dt * (rotER + dfdR(P)), -dt * (rotEz + dfdz(P)), -dt * (rotEf + 0.0),
               -dt * p["ch2"] * divB - pp / p["tau"])
        for f in range(7):
            bx(dU[f])[...] = As * bx(dU[f]) + rhs[f]
        for f in range(7):
            bx(U[f])[...] = bx(U[f]) + Bs * bx(dU[f])

    def clamps():
        """kernel_Epar_thread / kernel_EgtB_thread (:236-294)."""
        E = [bx(U[c]) for c in range(3)]
        B = [bx(U[3 + c]) for c in range(3)]
        if p["clean_ep"]:
            B2 = np.maximum(B[0] ** 2 + B[1] ** 2 + B[2] ** 2, TN)
            EB = E[0] * B[0] + E[1] * B[1] + E[2] * B[2]
            for c in range(3):
                E[c][...] = E[c] - EB / B2 * B[c]
        if p["check_egb"]:
            B2 = np.maximum(B[0] ** 2 + B[1] ** 2 + B[2] ** 2, TN)
            E2 = E[0] ** 2 + E[1] ** 2 + E[2] ** 2
            with np.errstate(invalid="ignore", divide="ignore"):
                s = np.where(E2 > B2, np.sqrt(B2 / E2), 1.0)
            for c in range(3):
                E[c][...] = np.where(E2 > B2, E[c] * s, E[c])

    def boundary_axis():
        """kernel_boundary_axis_thread (:371-411), on the R = 0 column."""
        cols = [i for i in range(bx.i0, bx.i1) if abs(Rv[i]) < dR / 4.0]
        j0, j1 = bx.j0, bx.j1
        for i in cols:
            for c, keep in ((0, 0), (1, 1), (2, 0), (3, 0), (4, 1), (5, 0), (6, 1)):
                U[c, j0:j1, i] = U[c, j0:j1, i + 1] if keep else 0.0
            for l in range(1, 4):
                for c, sgn in ((0, -1), (1, 1), (2, -1), (3, -1), (4, 1), (5, -1), (6, 1)):
                    U[c, j0:j1, i - l] = sgn * U[c, j0:j1, i + l]

    def wpert(t, R, z):
        """wpert (:413-443)."""
        th1 = math.acos(math.sqrt(1.0 - 1.0 / p["rpert1"]))
        th2 = math.acos(math.sqrt(1.0 - 1.0 / p["rpert2"]))
        if th1 > th2:
            th1, th2 = th2, th1
        r = np.sqrt(R * R + z * z)
        with np.errstate(invalid="ignore", divide="ignore"):
            th = np.arccos(z / r)
        mu = (th1 + th2) / 2.0
        s = (mu - th1) / 3.0
        if not (p["tp_start"] <= t <= p["tp_end"]):
            return np.zeros_like(R)
        val = (p["dw0"] * np.exp(-0.5 * ((th - mu) / s) ** 2)
               * math.sin((t - p["tp_start"]) * 2.0 * math.pi / (p["tp_end"] - p["tp_start"]))
               * 0.5 * (1.0 + np.tanh((r - 0.5 * radius) / (0.05 * radius))))
        with np.errstate(invalid="ignore"):
            return np.where((th >= th1) & (th <= th2), val, 0.0)

    def boundary_pulsar(t):
        """kernel_boundary_pulsar_thread (:445-530)."""
        R, z = Rb, Zb
        r2 = np.maximum(R * R + z * z, TN)
        r = np.sqrt(r2)
        on = r < 2.0 * radius
        ri = 0.5 * radius
        sB, sEperp, sEpar = 0.5 * dR, 0.25 * dR, 0.5 * dR
        d1 = 4 * dR
        rr = np.sqrt(R * R + z * z)
        rr = np.where(np.abs(rr) < TN, TN, rr)
        xn, zn = R / rr, z / rr
        m = b0 * radius ** 3
        bRn = m * ((3.0 * xn * zn) / (rr ** 3 + TN))
        bzn = m * ((3.0 * zn * zn - 1.0) / (rr ** 3 + TN))
        ER, Ez, Ef, BR, Bz, Bf = (bx(U[c]) for c in range(6))
        shape = lambda r0, d: 0.5 * (1.0 - np.tanh((r - r0) / d))  # noqa: E731
        s = shape(radius - d1, sB)
        bnp, bp = bRn * R + bzn * z, BR * R + Bz * z
        BRn = bnp * R / r2 * s + bp * R / r2 * (1 - s)
        Bzn = bnp * z / r2 * s + bp * z / r2 * (1 - s)
        BRn = BRn + (bRn - bnp * R / r2) * s + (BR - bp * R / r2) * (1 - s)
        Bzn = Bzn + (bzn - bnp * z / r2) * s + (Bz - bp * z / r2) * (1 - s)
        Bfn = 0.0 * s + Bf * (1 - s)
        w = p["omega"] + wpert(t, R, z)
        eRn, ezn = -w * R * Bz, w * R * BR
        enp, ep = eRn * R + ezn * z, ER * R + Ez * z
        s = shape(radius, sEperp)
        ERn = enp * R / r2 * s + ep * R / r2 * (1 - s)
        Ezn = enp * z / (r * r) * s + ep * z / r2 * (1 - s)
        s = shape(radius, sEpar)
        ERn = ERn + (eRn - enp * R / r2) * s + (ER - ep * R / r2) * (1 - s)
        Ezn = Ezn + (ezn - enp * z / r2) * s + (Ez - ep * z / r2) * (1 - s)
        Efn = 0.0 * s + Ef * (1 - s)
        core = on & (r < ri)
        new = [np.where(core, eRn, ERn), np.where(core, ezn, Ezn), np.where(core, 0.0, Efn),
               np.where(core, bRn, BRn), np.where(core, bzn, Bzn), np.where(core, 0.0, Bfn)]
        for c in range(6):
            u = bx(U[c])
            u[...] = np.where(on, new[c], u)

    def boundary_absorbing(Un):
        """kernel_boundary_absorbing_cylindrical (:532-591)."""
        xh = p["lower"][0] + p["size"][0] - p["pml"][0] * dR
        xl = -xh
        yh = p["lower"][1] + p["size"][1] - p["pml"][1] * dz
        yl = p["lower"][1] + p["pml"][1] * dz
        scale = p["pmllen"] * dR
        R, z = Rb, Zb
        sig = _pmlsigma(R, xl, xh, scale, p["sigpml"]) + _pmlsigma(z, yl, yh, scale, p["sigpml"])
        on = ((R > xh) | (z < yl) | (z > yh)) & (sig > TN)
        with np.errstate(invalid="ignore", divide="ignore"):
            ex = np.exp(-sig)
            fac = np.where(on, (1.0 - ex) / np.where(on, sig, 1.0), 0.0)
        for c in range(6):
            u, un = bx(U[c]), bx(Un[c])
            u[...] = np.where(on, ex * un + fac * (u - un), u)

    def ko():
        """kernel_KO_step1_thread / _step2_thread (:297-369)."""
        tmp = [_d6(U[f], bx, 0) + _d6(U[f], bx, 1) for f in range(7)]
        for f in range(7):
            bx(U[f])[...] = bx(U[f]) - p["KOeps"] * KO_CONST * tmp[f]

    time = T(time0)
    for _ in range(nsteps):
        Un = U.copy()
        for s in range(5):
            rk_stage(T(AS[s]), T(BS[s]))
            clamps()
            boundary_axis()
            boundary_pulsar(time + T(CS_CYL[s]) * dt)
            if s == 4:
                boundary_absorbing(Un)
            _periodic_fill(U, pl)
        ko()
        clamps()
        boundary_axis()
        boundary_pulsar(time + dt)
        _periodic_fill(U, pl)
        time = T(time + dt)
    return U
