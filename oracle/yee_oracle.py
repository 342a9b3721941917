"""numpy restatement of the reference's staggered (Yee) RK3 solver.

TEST INFRASTRUCTURE ONLY: the checker for the staggered kernels of
coffee_b200.  Nothing in the library imports this module.

  yee_evolve   field_solver::evolve_fields (src/algorithms/field_solver.cu:690-726)
  _push        kernel_compute_rho_thread + kernel_rk_push_thread (:22-152)
  update       kernel_rk_update_thread (:154-184)
  _clean_epar  kernel_clean_epar_thread (:186-262)
  _check_egb   kernel_check_eGTb_thread (:264-342)
  _pulsar_b/_e kernel_boundary_pulsar_{B,E}_thread (:344-638)
  _absorbing   kernel_boundary_absorbing_thread (src/algorithms/boundary.cu:18-78)
  interp       interpolate (src/algorithms/interpolation.h:9-33)
  gryee_evolve field_solver_gr::evolve_fields_gr, the staggered solver in
               Cartesian Kerr-Schild coordinates (src/algorithms/field_solver_gr.cu:810-861)

Layout (src/data/sim_data.cpp:19-25): Stagger bit a set means "on the grid
vertex along axis a", clear means "half a cell above it" (Grid::pos,
src/data/grid.h:103-134).  E_x is 0b110 (at (i+1/2, j, k)), E_y 0b101,
E_z 0b011, B_x 0b001 (at (i, j+1/2, k+1/2)), B_y 0b010, B_z 0b100, the
charge density 0b111.  Arrays are (d2, d1, d0), i fastest.

Every kernel of the reference runs over the box [guard - shift, dims -
guard + shift) of every axis; here each one is applied to the whole box at
once from slices shifted by its offsets.  Three properties of the reference
that matter for parity:

* rho is a solver array written only inside the box and zero elsewhere, so
  the currents of the last box cell along an axis see rho = 0 beyond it.
* kernel_check_eGTb_thread reads E through interpolation while it rewrites
  E in place, a race between threads of the GPU build.  This restatement
  reads the E of before the kernel everywhere (the order-free reading);
  the two agree wherever no neighbour is rescaled, i.e. wherever |E| <= |B|
  around the point.
* the pulsar boundary copies its whole scratch arrays back (copy_from), so
  after it every E and B point outside the box holds 0 until the guard
  exchange refills the periodic ones.
"""
from __future__ import annotations

import numpy as np

try:
    from .axisym_oracle import as_dict, tiny
    from .gr_oracle import Cks
except ImportError:  # imported as a top-level module
    from axisym_oracle import as_dict, tiny
    from gr_oracle import Cks

ST_E = (0b110, 0b101, 0b011)
ST_B = (0b001, 0b010, 0b100)
ST_RHO = 0b111
# SSP-RK3 in the form E = c1 En + c2 E + c3 dE (field_solver.cu:694-718)
RK3 = ((1.0, 0.0, 1.0, 1.0), (0.75, 0.25, 0.25, 0.5), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 1.0))


class Geo:
    """Grid of one rank in the reference's Scalar arithmetic."""

    def __init__(self, p, dtype):
        p = as_dict(p)
        ft = np.dtype(dtype).type
        self.ft = ft
        self.N = [int(n) for n in p["N"]]
        self.g = [int(g) for g in p["guard"]]
        self.d = [self.N[a] + 2 * self.g[a] for a in range(3)]
        self.delta = [ft(ft(p["size"][a]) / ft(self.N[a])) for a in range(3)]
        self.inv = [ft(ft(1.0) / self.delta[a]) for a in range(3)]
        self.lower = [ft(p["lower"][a]) for a in range(3)]
        self.size = [ft(p["size"][a]) for a in range(3)]
        s = int(p.get("shift_ghost", 0))
        self.lo = [self.g[a] - s for a in range(3)]
        self.hi = [self.d[a] - self.g[a] + s for a in range(3)]
        self.periodic = [bool(x) for x in p["periodic_boundary"]]

    def boxed(self, lo, hi):
        """The same grid with another box (e.g. the E, H box [1, dims - 1))."""
        g = Geo.__new__(Geo)
        g.__dict__.update(self.__dict__)
        g.lo, g.hi = list(lo), list(hi)
        return g

    def S(self, f, dz=0, dy=0, dx=0):
        """f over the box shifted by (dz, dy, dx)."""
        return f[self.lo[2] + dz:self.hi[2] + dz, self.lo[1] + dy:self.hi[1] + dy,
                 self.lo[0] + dx:self.hi[0] + dx]

    def pos(self, axis, stagger):
        """Grid::pos(axis, n, stagger) of the box points along `axis`, shaped to
        broadcast over the box (stagger 1: vertex, 0: half a cell above)."""
        ft = self.ft
        n = np.arange(self.lo[axis], self.hi[axis])
        cell = (n - self.g[axis]).astype(ft) + ft(0.0 if stagger else 0.5)
        v = self.lower[axis] + self.delta[axis] * cell
        shape = [1, 1, 1]
        shape[2 - axis] = -1
        return v.reshape(shape)


def interp(G: Geo, f, st_in: int, st_out: int):
    """interpolate(f, ijk, in, out) over the box: the average of the 1, 2, 4 or
    8 points of stagger `st_in` around each point of stagger `st_out`, summed
    pairwise along z, then y, then x (interpolation.h:9-33)."""
    def offs(a):
        i, o = (st_in >> a) & 1, (st_out >> a) & 1
        return (0, 0) if i == o else (-o, 1 - o)
    im, ip = offs(0)
    jm, jp = offs(1)
    km, kp = offs(2)
    h = G.ft(0.5)
    f11 = h * (G.S(f, km, jp, ip) + G.S(f, kp, jp, ip))
    f10 = h * (G.S(f, km, jm, ip) + G.S(f, kp, jm, ip))
    f01 = h * (G.S(f, km, jp, im) + G.S(f, kp, jp, im))
    f00 = h * (G.S(f, km, jm, im) + G.S(f, kp, jm, im))
    return h * (h * (f11 + f10) + h * (f01 + f00))


def _push(G: Geo, p, E, B, B0, rho, dE, dB):
    ft = G.ft
    T = ft(tiny(ft))
    S = G.S
    rho[:] = 0
    G.S(rho)[...] = (G.inv[0] * (S(E[0]) - S(E[0], 0, 0, -1)) +
                     G.inv[1] * (S(E[1]) - S(E[1], 0, -1, 0)) +
                     G.inv[2] * (S(E[2]) - S(E[2], -1, 0, 0)))
    dt = ft(p["dt"])
    CCx, CCy, CCz = (dt * G.inv[a] for a in range(3))
    ex, ey, ez = E
    bx, by, bz = B
    S(dB[0])[...] = CCz * (S(ey, 1) - S(ey)) - CCy * (S(ez, 0, 1) - S(ez))
    S(dB[1])[...] = CCx * (S(ez, 0, 0, 1) - S(ez)) - CCz * (S(ex, 1) - S(ex))
    S(dB[2])[...] = CCy * (S(ex, 0, 1) - S(ex)) - CCx * (S(ey, 0, 0, 1) - S(ey))

    def curlb(b):
        x, y, z = b
        return ((CCz * (S(y, -1) - S(y)) - CCy * (S(z, 0, -1) - S(z))),
                (CCx * (S(z, 0, 0, -1) - S(z)) - CCz * (S(x, -1) - S(x))),
                (CCy * (S(x, 0, -1) - S(x)) - CCx * (S(y, 0, 0, -1) - S(y))))
    cb, cb0 = curlb(B), curlb(B0)
    for a in range(3):
        out = ST_E[a]
        ir = interp(G, rho, ST_RHO, out)
        ie = [interp(G, E[c], ST_E[c], out) for c in range(3)]
        ib = [interp(G, B[c], ST_B[c], out) for c in range(3)]
        b2 = ib[0] * ib[0] + ib[1] * ib[1] + ib[2] * ib[2] + T
        cross = (ie[(a + 1) % 3] * ib[(a + 2) % 3] - ib[(a + 1) % 3] * ie[(a + 2) % 3])
        j = dt * ir * cross / b2
        S(dE[a])[...] = (cb[a] - cb0[a]) - j


def _update(G: Geo, U, Un, dU, c1, c2, c3):
    ft = G.ft
    c1, c2, c3 = ft(c1), ft(c2), ft(c3)
    for a in range(len(U)):
        G.S(U[a])[...] = c1 * G.S(Un[a]) + c2 * G.S(U[a]) + c3 * G.S(dU[a])


def _clean_epar(G: Geo, E, B, dE):
    T = G.ft(tiny(G.ft))
    for a in range(3):
        out = ST_E[a]
        ie = [interp(G, E[c], ST_E[c], out) for c in range(3)]
        ib = [interp(G, B[c], ST_B[c], out) for c in range(3)]
        dot = ie[0] * ib[0] + ie[1] * ib[1] + ie[2] * ib[2]
        G.S(dE[a])[...] = G.S(E[a]) - dot * ib[a] / (ib[0] * ib[0] + ib[1] * ib[1] +
                                                     ib[2] * ib[2] + T)


def _check_egb(G: Geo, E, B, dE):
    """E = temp * dE with temp = sqrt(B^2 / E^2) where E^2 > B^2, both
    interpolated to the component's position from the E of before the call."""
    ft, T = G.ft, G.ft(tiny(G.ft))
    temps = []
    for a in range(3):
        out = ST_E[a]
        ie = [interp(G, E[c], ST_E[c], out) for c in range(3)]
        ib = [interp(G, B[c], ST_B[c], out) for c in range(3)]
        emag = ie[0] * ie[0] + ie[1] * ie[1] + ie[2] * ie[2] + T
        bmag = ib[0] * ib[0] + ib[1] * ib[1] + ib[2] * ib[2] + T
        with np.errstate(invalid="ignore", divide="ignore"):
            temps.append(np.where(emag > bmag, np.sqrt(bmag / emag), ft(1.0)).astype(ft))
    for a in range(3):
        G.S(E[a])[...] = temps[a] * G.S(dE[a])


def _pmlsigma(x, xl, xh, scale, sig0):
    """pmlsigma (src/algorithms/boundary.cu:7-15)."""
    qh = (x - xh) / scale
    ql = (xl - x) / scale
    return np.where(x > xh, sig0 * (qh * qh * qh), np.where(x < xl, sig0 * (ql * ql * ql), 0))


def _absorbing(G: Geo, p, U, Un):
    ft, T = G.ft, G.ft(tiny(G.ft))
    x, y, z = (G.pos(a, 1) for a in range(3))
    pml = p["pml"]
    hi = [G.lower[a] + G.size[a] - ft(pml[a]) * G.delta[a] for a in range(3)]
    lo = [G.lower[a] + ft(pml[a]) * G.delta[a] for a in range(3)]
    scale = ft(p["pmllen"]) * G.delta[0]
    sig0 = ft(p["sigpml"])
    outside = ((x > hi[0]) | (x < lo[0]) | (y > hi[1]) | (y < lo[1]) | (z > hi[2]) | (z < lo[2]))
    sig = (_pmlsigma(x, lo[0], hi[0], scale, sig0) + _pmlsigma(y, lo[1], hi[1], scale, sig0) +
           _pmlsigma(z, lo[2], hi[2], scale, sig0)).astype(ft)
    sig = np.broadcast_to(sig, G.S(U[0]).shape)
    act = np.broadcast_to(outside, sig.shape) & (sig > T)
    if not act.any():
        return
    s = np.where(act, sig, ft(1.0))
    e = np.exp(-s)
    for a in range(len(U)):
        u, un = G.S(U[a]), G.S(Un[a])
        new = (e * un).astype(np.float64) + (1.0 - e.astype(np.float64)) / s.astype(
            np.float64) * (u - un).astype(np.float64)
        u[...] = np.where(act, new.astype(ft), u)


def _star(p, G: Geo, x, y, z, phase):
    """b0 * quadru_dipole(x, y, z, ..., phase, n) for n = 0, 1, 2
    (src/algorithms/pulsar_impl.hpp:57-129) in the reference's Scalar
    arithmetic: the terms with a double literal are evaluated in float64 and
    rounded to Scalar on return, as C++ promotes them."""
    ft = G.ft
    f8 = np.float64
    T = ft(tiny(ft))
    c, s = np.cos(phase), np.sin(phase)
    p1, p2, p3 = ft(p["p1"]), ft(p["p2"]), ft(p["p3"])
    p1t, p2t, p3t = p1 * c - p2 * s, p1 * s + p2 * c, p3
    r2 = x * x + y * y + z * z
    pr = (p1t * x + p2t * y + p3t * z).astype(f8)
    den = (np.sqrt(r2 * r2 * r2) + T).astype(f8)
    r2t = (r2 + T).astype(f8)
    dip = [((3.0 * q.astype(f8) * pr / r2t - f8(pq)) / den).astype(ft)
           for q, pq in ((x, p1t), (y, p2t), (z, p3t))]
    q11, q12, q13 = ft(p["q11"]), ft(p["q12"]), ft(p["q13"])
    q22, q23 = ft(p["q22"]), ft(p["q23"])
    c8, s8 = f8(c), f8(s)
    q11t = ft(f8(q11 * (c * c)) - 2.0 * f8(q12) * c8 * s8 + f8(q22 * (s * s)))
    q12t = ft(f8(q12) * np.cos(2.0 * f8(phase)) + f8((q11 - q22) * c * s))
    q22t = ft(f8(q22 * (c * c)) + f8(q11 * (s * s)) + 2.0 * f8(q12) * c8 * s8)
    q13t = q13 * c - q23 * s
    q23t = q23 * c + q13 * s
    q33t = -q11 - q22
    ox = ft(p["q_offset_x"]) * c - ft(p["q_offset_y"]) * s
    oy = ft(p["q_offset_x"]) * s + ft(p["q_offset_y"]) * c
    x1, y1, z1 = x - ox, y - oy, z - ft(p["q_offset_z"])
    q2 = x1 * x1 + y1 * y1 + z1 * z1
    r7 = (q2 * q2 * q2 * np.sqrt(q2) + T).astype(f8)
    X1, Y1, Z1 = x1.astype(f8), y1.astype(f8), z1.astype(f8)
    xqx = (f8(q11t) * X1 * X1 + 2.0 * f8(q12t) * X1 * Y1 + f8(q22t) * Y1 * Y1 +
           2.0 * (q13t * x1 + q23t * y1).astype(f8) * Z1 + f8(q33t) * Z1 * Z1).astype(ft)
    xqx = xqx.astype(f8)
    Q2 = q2.astype(f8)
    quad = [((-2.0 * (q11t * x1 + q12t * y1 + q13t * z1).astype(f8) * Q2 + 5.0 * X1 * xqx) /
             r7).astype(ft),
            ((-2.0 * (q12t * x1 + q22t * y1 + q23t * z1).astype(f8) * Q2 + 5.0 * Y1 * xqx) /
             r7).astype(ft),
            ((-2.0 * (q13t * x1 + q23t * y1 + q33t * z1).astype(f8) * Q2 + 5.0 * Z1 * xqx) /
             r7).astype(ft)]
    b0 = ft(p["b0"])
    return [b0 * (dip[n] + quad[n]) for n in range(3)]


def _shape(G: Geo, r, r0, d):
    """shape (src/algorithms/pulsar_impl.hpp:52-55); the GPU build evaluates
    tanh in Scalar."""
    return (0.5 * (1.0 - np.tanh((r - r0) / d).astype(np.float64))).astype(G.ft)


def _blend(v_star, v_in, pos, r2, a, s_perp, s_par):
    """Component `a` of the reference's star blend: the radial part from the
    star field with weight s_perp, the rest with weight s_par."""
    rad_s = (v_star[0] * pos[0] + v_star[1] * pos[1] + v_star[2] * pos[2]) * pos[a] / r2
    rad_i = (v_in[0] * pos[0] + v_in[1] * pos[1] + v_in[2] * pos[2]) * pos[a] / r2
    out = rad_s * s_perp + rad_i * (1 - s_perp)
    out = out + ((v_star[a] - rad_s) * s_par + (v_in[a] - rad_i) * (1 - s_par))
    return out


def _pulsar_b(G: Geo, p, B, t):
    ft = G.ft
    x0, y0, z0 = (G.pos(a, 1) for a in range(3))
    rl = ft(2.0 * ft(p["radius"]))
    mask = np.broadcast_to(x0 * x0 + y0 * y0 + z0 * z0 < rl * rl, G.S(B[0]).shape)
    d1 = ft(4) * G.delta[0]
    sc = ft(1.0) * G.delta[0]
    phase = ft(p["omega"]) * ft(t)
    out = []
    for a in range(3):
        st = ST_B[a]
        pos = [G.pos(c, (st >> c) & 1) for c in range(3)]
        pos = [np.broadcast_to(q, mask.shape) for q in pos]
        r2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]
        r = np.sqrt(r2)
        star = _star(p, G, pos[0], pos[1], pos[2], phase)
        vin = [G.S(B[c]) if c == a else interp(G, B[c], ST_B[c], st) for c in range(3)]
        s = _shape(G, r, ft(p["radius"]) - d1, sc)
        new = _blend(star, vin, pos, r2, a, s, s)
        out.append(np.where(mask, new, G.S(B[a])))
    return out


def _pulsar_e(G: Geo, p, E, B, t):
    ft = G.ft
    x0, y0, z0 = (G.pos(a, 1) for a in range(3))
    rl = ft(2.0 * ft(p["radius"]))
    mask = np.broadcast_to(x0 * x0 + y0 * y0 + z0 * z0 < rl * rl, G.S(E[0]).shape)
    s_par = ft(1.0) * G.delta[0]
    s_perp = ft(0.5) * G.delta[0]
    w = ft(p["omega"])
    out = []
    for a in range(3):
        st = ST_E[a]
        pos = [np.broadcast_to(G.pos(c, (st >> c) & 1), mask.shape) for c in range(3)]
        r2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]
        r = np.sqrt(r2)
        vx, vy = -w * pos[1], w * pos[0]
        ie = [interp(G, E[c], ST_E[c], st) for c in range(3)]
        ib = [interp(G, B[c], ST_B[c], st) for c in range(3)]
        star = [-vy * ib[2], vx * ib[2], -vx * ib[1] + vy * ib[0]]
        r0 = ft(p["radius"]) - ft(0)
        sp = _shape(G, r, r0, s_perp)
        sq = _shape(G, r, r0, s_par)
        new = _blend(star, ie, pos, r2, a, sp, sq)
        out.append(np.where(mask, new, G.S(E[a])))
    return out


def _exchange(G: Geo, U):
    """Single-rank guard exchange of the periodic axes, x then y then z
    (src/sim_env_impl.hpp:180-195 with both neighbours = self)."""
    for a in range(3):
        if not G.periodic[a]:
            continue
        g, n = G.g[a], G.N[a]
        ax = 2 - a
        for f in U:
            idx_dst = [slice(None)] * 3
            idx_src = [slice(None)] * 3
            idx_dst[ax], idx_src[ax] = slice(n + g, n + 2 * g), slice(g, 2 * g)
            f[tuple(idx_dst)] = f[tuple(idx_src)]
            idx_dst[ax], idx_src[ax] = slice(0, g), slice(n, n + g)
            f[tuple(idx_dst)] = f[tuple(idx_src)]


def yee_evolve(p, U: np.ndarray, nsteps: int, time0: float = 0.0, B0=None):
    """Advance U = (Ex, Ey, Ez, Bx, By, Bz[, P]) (arrays (d2, d1, d0)) by nsteps
    evolve_fields calls of the reference's staggered solver, starting at
    time0 and advancing time by dt in the dtype of U.  B0 is the background
    field subtracted in the curl of B (zero when None).  P is left alone."""
    p = as_dict(p)
    U = np.array(U, copy=True)
    ft = U.dtype.type
    G = Geo(p, U.dtype)
    E, B = U[0:3], U[3:6]
    B0 = np.zeros_like(B) if B0 is None else np.asarray(B0, dtype=U.dtype)
    rho = np.zeros_like(E[0])
    dt = ft(p["dt"])
    t = ft(time0)
    for _ in range(nsteps):
        En, Bn = E.copy(), B.copy()
        dE, dB = np.zeros_like(E), np.zeros_like(B)
        for sub, (c1, c2, c3, tf) in enumerate(RK3):
            last = sub == 2
            _push(G, p, E, B, B0, rho, dE, dB)
            _update(G, E, En, dE, c1, c2, c3)
            for a in range(3):
                G.S(dE[a])[...] = G.S(E[a])
            _update(G, B, Bn, dB, c1, c2, c3)
            if last:
                _clean_epar(G, E, B, dE)
            _check_egb(G, E, B, dE)
            if p["problem"] == 1:
                # t + dt in Scalar; t + 0.5 * dt through double (field_solver.cu:694-717)
                tb = ft(t + dt) if tf == 1.0 else ft(np.float64(t) + 0.5 * np.float64(dt))
                nb = _pulsar_b(G, p, B, tb)
                for a in range(3):
                    G.S(dB[a])[...] = nb[a]
                B[...] = dB
                ne = _pulsar_e(G, p, E, B, tb)
                for a in range(3):
                    G.S(dE[a])[...] = ne[a]
                E[...] = dE
            if last:
                _absorbing(G, p, U[0:6], np.concatenate([En, Bn]))
            _exchange(G, list(E) + list(B))
        t = ft(t + dt)
    return U


# ----------------------------------------------------------------- GR (Kerr-Schild)
# sim_data's E holds the densitised D.  E = alpha D_i + sqrt(gamma) (beta x B)_i
# and H = alpha B_i - sqrt(gamma) (beta x D)_i at the E and B positions, the
# lowered B (kept in sim_data's B0 by the reference) at the B positions.

def _cks_at(G: Geo, a, st, T):
    return Cks(a, G.pos(0, st & 1), G.pos(1, (st >> 1) & 1), G.pos(2, (st >> 2) & 1), T)


def _gr_eh(GE: Geo, a, T, D, B, Ed, Hd, Bd):
    """kernel_compute_E_gr_thread / kernel_compute_H_gr_thread
    (field_solver_gr.cu:81-225) over [1, dims - 1)."""
    for A in range(3):
        st = ST_E[A]
        m = _cks_at(GE, a, st, T)
        iD = [GE.S(D[c]) if c == A else interp(GE, D[c], ST_E[c], st) for c in range(3)]
        iB = [None if c == A else interp(GE, B[c], ST_B[c], st) for c in range(3)]
        dd = m.lower(iD)[A]
        b, c = (A + 1) % 3, (A + 2) % 3
        GE.S(Ed[A])[...] = m.alpha * dd + m.sqrt_gamma * (m.beta_u[b] * iB[c] -
                                                          m.beta_u[c] * iB[b])
    for A in range(3):
        st = ST_B[A]
        m = _cks_at(GE, a, st, T)
        iB = [GE.S(B[c]) if c == A else interp(GE, B[c], ST_B[c], st) for c in range(3)]
        iD = [None if c == A else interp(GE, D[c], ST_E[c], st) for c in range(3)]
        bd = m.lower(iB)[A]
        b, c = (A + 1) % 3, (A + 2) % 3
        GE.S(Hd[A])[...] = m.alpha * bd - m.sqrt_gamma * (m.beta_u[b] * iD[c] -
                                                          m.beta_u[c] * iD[b])
        GE.S(Bd[A])[...] = bd


def _gr_rho(G: Geo, a, T, D, rho):
    """kernel_compute_rho_gr_thread (field_solver_gr.cu:29-53): the
    sqrt(gamma)-weighted divergence of D at the vertices."""
    ft = G.ft
    x, y, z = (G.pos(c, 1) for c in range(3))
    h = [ft(G.delta[c] / 2.0) for c in range(3)]

    def sg(xx, yy, zz):
        return Cks(a, xx, yy, zz, T).sqrt_gamma
    rho[:] = 0
    G.S(rho)[...] = (G.inv[0] * (G.S(D[0]) * sg(x + h[0], y, z) - G.S(D[0], 0, 0, -1) *
                                 sg(x - h[0], y, z)) +
                     G.inv[1] * (G.S(D[1]) * sg(x, y + h[1], z) - G.S(D[1], 0, -1, 0) *
                                 sg(x, y - h[1], z)) +
                     G.inv[2] * (G.S(D[2]) * sg(x, y, z + h[2]) - G.S(D[2], -1, 0, 0) *
                                 sg(x, y, z - h[2]))) / sg(x, y, z)


def _gr_push(G: Geo, p, a, T, Ed, Hd, B, Bd, rho, dD, dB):
    """kernel_rk_push_gr_thread (field_solver_gr.cu:227-378)."""
    ft = G.ft
    S = G.S
    dt = ft(p["dt"])
    CCx, CCy, CCz = (dt * G.inv[c] for c in range(3))
    ex, ey, ez = Ed
    hx, hy, hz = Hd
    sgB = [_cks_at(G, a, ST_B[c], T).sqrt_gamma for c in range(3)]
    sgE = [_cks_at(G, a, ST_E[c], T).sqrt_gamma for c in range(3)]
    S(dB[0])[...] = (CCz * (S(ey, 1) - S(ey)) - CCy * (S(ez, 0, 1) - S(ez))) / sgB[0]
    S(dB[1])[...] = (CCx * (S(ez, 0, 0, 1) - S(ez)) - CCz * (S(ex, 1) - S(ex))) / sgB[1]
    S(dB[2])[...] = (CCy * (S(ex, 0, 1) - S(ex)) - CCx * (S(ey, 0, 0, 1) - S(ey))) / sgB[2]
    S(dD[0])[...] = (CCz * (S(hy, -1) - S(hy)) - CCy * (S(hz, 0, -1) - S(hz))) / sgE[0]
    S(dD[1])[...] = (CCx * (S(hz, 0, 0, -1) - S(hz)) - CCz * (S(hx, -1) - S(hx))) / sgE[1]
    S(dD[2])[...] = (CCy * (S(hx, 0, -1) - S(hx)) - CCx * (S(hy, 0, 0, -1) - S(hy))) / sgE[2]
    if not p.get("calc_current", True):
        return
    for A in range(3):
        out = ST_E[A]
        ir = interp(G, rho, ST_RHO, out)
        ie = [interp(G, Ed[c], ST_E[c], out) for c in range(3)]
        ib = [interp(G, B[c], ST_B[c], out) for c in range(3)]
        ibd = [interp(G, Bd[c], ST_B[c], out) for c in range(3)]
        b, c = (A + 1) % 3, (A + 2) % 3
        cross = ie[b] * ibd[c] - ibd[b] * ie[c]
        den = ib[0] * ibd[0] + ib[1] * ibd[1] + ib[2] * ibd[2] + T
        S(dD[A])[...] = S(dD[A]) - dt * ir * cross / sgE[A] / den


def _gr_clean(G: Geo, a, T, D, B, dD):
    """kernel_clean_epar_gr_thread (field_solver_gr.cu:416-517)."""
    for A in range(3):
        st = ST_E[A]
        m = _cks_at(G, a, st, T)
        iD = [G.S(D[c]) if c == A else interp(G, D[c], ST_E[c], st) for c in range(3)]
        iB = [interp(G, B[c], ST_B[c], st) for c in range(3)]
        bd = m.lower(iB)
        dot = iD[0] * bd[0] + iD[1] * bd[1] + iD[2] * bd[2]
        den = iB[0] * bd[0] + iB[1] * bd[1] + iB[2] * bd[2] + T
        G.S(dD[A])[...] = G.S(D[A]) - dot * iB[A] / den


def _gr_check(G: Geo, a, T, dD, B, D):
    """kernel_check_eGTb_gr_thread (field_solver_gr.cu:519-647): reads dD
    and B, writes D, so it is free of the flat solver's race."""
    ft = G.ft
    out = []
    for A in range(3):
        st = ST_E[A]
        m = _cks_at(G, a, st, T)
        iD = [G.S(dD[c]) if c == A else interp(G, dD[c], ST_E[c], st) for c in range(3)]
        dd = m.lower(iD)
        emag = iD[0] * dd[0] + iD[1] * dd[1] + iD[2] * dd[2] + T
        iB = [interp(G, B[c], ST_B[c], st) for c in range(3)]
        bd = m.lower(iB)
        bmag = iB[0] * bd[0] + iB[1] * bd[1] + iB[2] * bd[2] + T
        with np.errstate(invalid="ignore", divide="ignore"):
            temp = np.where(emag > bmag, np.sqrt(bmag / emag), ft(1.0)).astype(ft)
        out.append(temp * G.S(dD[A]))
    for A in range(3):
        G.S(D[A])[...] = out[A]


def _gr_absorbing(G: Geo, p, a, T, U, Un):
    """kernel_absorbing_boundary_gr_thread (field_solver_gr.cu:661-775): the
    damping layer inside 0.8 r_H (rate sig0 cube((r1 - r) / (0.2 r_H)) dt at
    each component's position), zero inside 0.01 r_H, the outer layer
    (pmlsigma_gr), and the start-of-step values on and beyond the box edge."""
    ft = G.ft
    f8 = np.float64
    x, y, z = (G.pos(c, 1) for c in range(3))
    shape = G.S(U[0]).shape
    rH = ft(1.0 + np.sqrt(1.0 - f8(a * a)))
    r1, r2, dd = ft(0.8 * f8(rH)), ft(0.01 * f8(rH)), ft(0.2 * f8(rH))
    sig0 = ft(p["sigpml"])
    dt = ft(p["dt"])
    h = [ft(G.delta[c] / 2.0) for c in range(3)]
    r = np.broadcast_to(Cks(a, x, y, z, T).r, shape)
    off = [(h[0], 0, 0), (0, h[1], 0), (0, 0, h[2]), (0, h[1], h[2]), (h[0], 0, h[2]),
           (h[0], h[1], 0)]
    for c in range(6):
        u, un = G.S(U[c]), G.S(Un[c])
        rc = Cks(a, x + ft(off[c][0]), y + ft(off[c][1]), z + ft(off[c][2]), T).r
        q = (r1 - rc) / dd
        sig = np.broadcast_to((sig0 * (q * q * q)) * dt, shape)
        act = (r < r1) & (sig > T)
        s = np.where(act, sig, ft(1.0))
        e = np.exp(-s)
        new = ((e * un).astype(f8) + (1.0 - e.astype(f8)) / s.astype(f8) *
               (u - un).astype(f8)).astype(ft)
        u[...] = np.where(act, new, u)
    for c in range(6):
        u = G.S(U[c])
        u[...] = np.where(r < r2, ft(0), u)
    pml = p["pml"]
    hi = [G.lower[c] + G.size[c] - ft(pml[c]) * G.delta[c] for c in range(3)]
    lo = [G.lower[c] + ft(pml[c]) * G.delta[c] for c in range(3)]
    scale = ft(p["pmllen"]) * G.delta[0]

    def ps(v, vl, vh):
        qh = ((v - vh) / scale).astype(f8)
        ql = ((vl - v) / scale).astype(f8)
        return np.where(v > vh, (f8(sig0) * qh ** 3.0).astype(ft),
                        np.where(v < vl, (f8(sig0) * ql ** 3.0).astype(ft), ft(0)))
    outside = np.broadcast_to((x > hi[0]) | (x < lo[0]) | (y > hi[1]) | (y < lo[1]) |
                              (z > hi[2]) | (z < lo[2]), shape)
    sig = np.broadcast_to((ps(x, lo[0], hi[0]) + ps(y, lo[1], hi[1]) + ps(z, lo[2], hi[2])
                           ).astype(ft), shape)
    act = outside & (sig > T)
    if act.any():
        s = np.where(act, sig, ft(1.0))
        e = np.exp(-s)
        for c in range(6):
            u, un = G.S(U[c]), G.S(Un[c])
            new = ((e * un).astype(f8) + (1.0 - e.astype(f8)) / s.astype(f8) *
                   (u - un).astype(f8)).astype(ft)
            u[...] = np.where(act, new, u)
    up = [G.lower[c] + G.size[c] for c in range(3)]
    edge = np.broadcast_to((x <= G.lower[0]) | (x >= up[0]) | (y <= G.lower[1]) |
                           (y >= up[1]) | (z <= G.lower[2]) | (z >= up[2]), shape)
    for c in range(6):
        u, un = G.S(U[c]), G.S(Un[c])
        u[...] = np.where(edge, un, u)


def gryee_evolve(p, U: np.ndarray, nsteps: int):
    """Advance U = (Dx, Dy, Dz, Bx, By, Bz[, P]) by nsteps
    field_solver_gr::evolve_fields_gr calls (field_solver_gr.cu:810-861):
    per substep E and H over [1, dims - 1), rho, push, update, then the
    E_par cleaning (last substep, clean_ep), the rescale (check_egb) and the
    absorbing layers (last substep).  The axes are not periodic."""
    p = as_dict(p)
    U = np.array(U, copy=True)
    ft = U.dtype.type
    T = ft(tiny(ft))
    G = Geo(p, U.dtype)
    GE = G.boxed([1, 1, 1], [d - 1 for d in G.d])
    a = ft(p["a"])
    D, B = U[0:3], U[3:6]
    Ed, Hd, Bd = np.zeros_like(D), np.zeros_like(B), np.zeros_like(B)
    rho = np.zeros_like(D[0])
    for _ in range(nsteps):
        Dn, Bn = D.copy(), B.copy()
        dD, dB = np.zeros_like(D), np.zeros_like(B)
        for sub, (c1, c2, c3, _tf) in enumerate(RK3):
            last = sub == 2
            _gr_eh(GE, a, T, D, B, Ed, Hd, Bd)
            _gr_rho(G, a, T, D, rho)
            _gr_push(G, p, a, T, Ed, Hd, B, Bd, rho, dD, dB)
            _update(G, D, Dn, dD, c1, c2, c3)
            for c in range(3):
                G.S(dD[c])[...] = G.S(D[c])
            _update(G, B, Bn, dB, c1, c2, c3)
            if last and p.get("clean_ep", True):
                _gr_clean(G, a, T, D, B, dD)
            if p.get("check_egb", True):
                _gr_check(G, a, T, dD, B, D)
            if last:
                _gr_absorbing(G, p, a, T, U[0:6], np.concatenate([Dn, Bn]))
    return U
