"""Initial conditions for the benchmark and test problems (host side, numpy).

These play the role of the reference's ``user_*.hpp`` snippets (e.g.
``src/user_alfven.hpp``, ``src/user_pulsar3d_EZ.hpp``): they fill E, B, P
on every grid point, guard cells included, at the collocated EZ vertex
positions ``lower + delta*(n - guard)`` (``Grid::pos`` with stagger bit 1,
``src/data/grid.h:116-134``).  Values are computed in float64 and returned
in the requested dtype, as 7 arrays of shape ``(d2, d1, d0)``.
"""
from __future__ import annotations

import math

import numpy as np

from .config import Grid, SimParams

# ---------------------------------------------------------------- Alfven wave


def alfven_params(N: int = 128, guard: int = 3) -> SimParams:
    """Periodic unit box, dx = 1/N, dt = 0.5*dx, no absorbing layer,
    no star (problem 0), E.B damping on (the reference default)."""
    p = SimParams()
    p.N = [N, N, N]
    p.guard = [guard] * 3
    p.lower = [0.0, 0.0, 0.0]
    p.size = [1.0, 1.0, 1.0]
    p.periodic_boundary = [True, True, True]
    p.pml = [0, 0, 0]
    p.problem = 0
    p.dt = 0.5 / N
    p.use_edotb_damping = True
    return p


def alfven_fields(p: SimParams, dtype=np.float32, amp=0.1, width2=0.02, vz=0.1):
    """B = (1, amp*sin(2 pi x)*exp(-((y-1/2)^2+(z-1/2)^2)/width2), 0),
    E = -v x B with v = vz zhat, so E = (vz*By, -vz*Bx, 0) and E.B = 0; P = 0."""
    g = Grid.from_params(p, dtype)
    ft = np.dtype(dtype)
    x = g.coords(0, np.float64)
    y = g.coords(1, np.float64)
    z = g.coords(2, np.float64)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    Bx = np.ones_like(X)
    By = amp * np.sin(2 * np.pi * X) * np.exp(-((Y - 0.5) ** 2 + (Z - 0.5) ** 2) / width2)
    Bz = np.zeros_like(X)
    Ex = vz * By
    Ey = -vz * Bx
    Ez = np.zeros_like(X)
    P = np.zeros_like(X)
    return [a.astype(ft) for a in (Ex, Ey, Ez, Bx, By, Bz, P)]


def _xyz(p: SimParams, dtype, stagger: int = 0b111):
    """Z, Y, X of every grid point at `stagger` (bit a set: the vertex along
    axis a, clear: half a cell above it; ``Grid::pos``, src/data/grid.h:103-134)."""
    g = Grid.from_params(p, dtype)
    c = [g.coords(a, np.float64) + (0.0 if (stagger >> a) & 1 else 0.5 * g.delta[a])
         for a in range(3)]
    return np.meshgrid(c[2], c[1], c[0], indexing="ij")


# Stagger of each component on the staggered (Yee) grid (src/data/sim_data.cpp:19-25)
YEE_STAGGER = (0b110, 0b101, 0b011, 0b001, 0b010, 0b100, 0b111)


def _per_component(fn, p: SimParams, dtype, yee: bool):
    """The 7 arrays fn(Z, Y, X, c) (c = 0..6: Ex Ey Ez Bx By Bz P, float64),
    each component taken at its own position on the staggered grid when
    `yee` (what vector_field::initialize does with the Yee staggering) or at
    the vertices otherwise."""
    ft = np.dtype(dtype)
    if not yee:
        Z, Y, X = _xyz(p, dtype)
        return [np.asarray(fn(Z, Y, X, c), dtype=ft) for c in range(7)]
    return [np.asarray(fn(*_xyz(p, dtype, st), c), dtype=ft) for c, st in enumerate(YEE_STAGGER)]


def alfven_plane_wave_fields(p: SimParams, dtype=np.float32, xi0=0.1, yee: bool = False):
    """Plane Alfven wave on B0 = x-hat in a periodic box, the initial
    condition of the reference's wave driver (``src/main-wave.cpp`` with
    ``src/user_alfven.hpp``): wave vector k = (2 * 2 pi / Lx, 0, 2 pi / Lz),
    frequency w = k.B0 / |B0| (c = 1), E along e = (k x B0) x B0 normalised,
    b = k x e, E = -xi0 sin(k.x) e, P = 0.  The EZ branch (collocated,
    every component at the vertices) sets B = B0 - xi0 sin(k.x) b / w.  With
    `yee`, the staggered branch: each E component at its own position and
    B = B0 + the staggered curl of A = xi0 cos(k.x) e / w taken at the E
    positions, so that B is divergence free on the grid
    (``src/user_alfven.hpp:79-113``; the last point of each axis, which the
    reference leaves unset, holds B0)."""
    b0 = np.array([1.0, 0.0, 0.0])
    k = np.array([2.0 * 2.0 * math.pi / p.size[0], 0.0, 1.0 * 2.0 * math.pi / p.size[2]])
    w = float(k @ b0) / float(np.linalg.norm(b0))
    e = np.cross(np.cross(k, b0), b0)
    e = e / np.linalg.norm(e)
    b = np.cross(k, e)

    def fn(Z, Y, X, c):
        if c == 6:
            return np.zeros_like(X)
        s = np.sin(k[0] * X + k[1] * Y + k[2] * Z)
        return -xi0 * s * e[c] if c < 3 else b0[c - 3] - xi0 * s * b[c - 3] / w
    if not yee:
        return _per_component(fn, p, dtype, False)
    ft = np.dtype(dtype)
    out = [np.asarray(fn(*_xyz(p, dtype, YEE_STAGGER[c]), c), dtype=ft) for c in range(3)]
    A = []
    for c in range(3):
        Z, Y, X = _xyz(p, dtype, YEE_STAGGER[c])
        A.append(xi0 * np.cos(k[0] * X + k[1] * Y + k[2] * Z) * e[c] / w)
    g = Grid.from_params(p, dtype)
    inv = g.inv_delta
    B = [np.full(A[0].shape, b0[c]) for c in range(3)]
    core = (slice(0, -1),) * 3
    sh = {0: (slice(0, -1), slice(0, -1), slice(1, None)),   # +x
          1: (slice(0, -1), slice(1, None), slice(0, -1)),   # +y
          2: (slice(1, None), slice(0, -1), slice(0, -1))}   # +z
    B[0][core] = b0[0] + (A[2][sh[1]] - A[2][core]) * inv[1] - (A[1][sh[2]] - A[1][core]) * inv[2]
    B[1][core] = b0[1] + (A[0][sh[2]] - A[0][core]) * inv[2] - (A[2][sh[0]] - A[2][core]) * inv[0]
    B[2][core] = b0[2] + (A[1][sh[0]] - A[1][core]) * inv[0] - (A[0][sh[1]] - A[0][core]) * inv[1]
    out += [np.asarray(a, dtype=ft) for a in B]
    out.append(np.zeros(A[0].shape, dtype=ft))
    return out


def emwave_fields(p: SimParams, dtype=np.float32, yee: bool = False):
    """Vacuum electromagnetic plane wave (``src/user_emwave.hpp``): k in the
    x-y plane, k = 2 pi (kn[0] / Lx, kn[1] / Ly), E = e sin(k.x) with the unit
    vector e in the x-y plane normal to k, B = z-hat sin(k.x), P = 0.  With
    `yee` each component is evaluated at its staggered position."""
    kx = p.kn[0] * 2.0 * math.pi / p.size[0]
    ky = p.kn[1] * 2.0 * math.pi / p.size[1]
    ex, ey = (1.0, -kx / ky) if ky != 0 else (-ky / kx, 1.0)
    nrm = math.hypot(ex, ey)
    ex, ey = ex / nrm, ey / nrm

    def fn(Z, Y, X, c):
        if c not in (0, 1, 5):
            return np.zeros_like(X)
        return {0: ex, 1: ey, 5: 1.0}[c] * np.sin(kx * X + ky * Y)
    return _per_component(fn, p, dtype, yee)


# ------------------------------------------------------------- turbulence

TURB_SEED = 20261203


def turbulence_params(N: int = 512, guard: int = 3, cfl: float = 0.5) -> SimParams:
    p = alfven_params(N, guard)
    p.dt = cfl / N
    return p


def turbulence_modes(seed: int = TURB_SEED, nmodes: int = 32, nmin: float = 2.0,
                     nmax: float = 8.0, db_rms: float = 0.3, nv: int = 8,
                     vmax_bound: float = 0.45):
    """Mode tables for the random force-free turbulence problem.

    A = sum_m a_m e_m cos(k_m.x + phi_m) with integer wave vectors n_m,
    |n_m| in [nmin, nmax], k = 2 pi n, e_m a random unit vector normal to k_m,
    so dB_m = curl A_m = -a_m (k_m x e_m) sin(k_m.x + phi_m).  Amplitudes
    follow |dB_m|^2 ~ |k_m|^-2 and are scaled so rms(dB) = db_rms (the modes
    are distinct and not opposite, so rms^2 = sum |dB_m|^2 / 2).

    v = sum_n c_n u_n sin(q_n.x + psi_n) with 1 <= |n| <= 2, unit u_n, and
    sum |c_n| = vmax_bound, which bounds |v| <= vmax_bound < 0.5.

    Returns float64 arrays: (kb[m,3], bamp[m,3], phib[m]), (kv, vamp, phiv),
    with bamp the vector amplitude of sin(k.x + phi) in dB.
    """
    rng = np.random.default_rng(seed)
    seen = set()
    ks, dirs = [], []
    while len(ks) < nmodes:
        n = rng.integers(-int(nmax), int(nmax) + 1, size=3)
        nn = float(np.linalg.norm(n))
        key = tuple(int(v) for v in n)
        neg = tuple(-v for v in key)
        if nn < nmin or nn > nmax or key in seen or neg in seen:
            continue
        seen.add(key)
        ks.append(n.astype(np.float64))
    kb = 2 * np.pi * np.array(ks)
    bamp = np.zeros((nmodes, 3))
    for m in range(nmodes):
        k = kb[m]
        e = rng.normal(size=3)
        e -= k * (e @ k) / (k @ k)
        e /= np.linalg.norm(e)
        kmag = np.linalg.norm(k)
        # a_m ~ |k|^-2  =>  |dB_m| = a_m |k| ~ |k|^-1
        a = kmag ** -2
        bamp[m] = -a * np.cross(k, e)
    phib = rng.uniform(0, 2 * np.pi, size=nmodes)
    rms = math.sqrt(0.5 * float(np.sum(bamp ** 2)))
    bamp *= db_rms / rms

    kvs = []
    seen = set()
    while len(kvs) < nv:
        n = rng.integers(-2, 3, size=3)
        nn = float(np.linalg.norm(n))
        key = tuple(int(v) for v in n)
        if nn < 1 or nn > 2 or key in seen:
            continue
        seen.add(key)
        kvs.append(n.astype(np.float64))
    kv = 2 * np.pi * np.array(kvs)
    u = rng.normal(size=(nv, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    c = rng.uniform(0.5, 1.0, size=nv)
    c *= vmax_bound / c.sum()
    vamp = u * c[:, None]
    phiv = rng.uniform(0, 2 * np.pi, size=nv)
    return (kb, bamp, phib), (kv, vamp, phiv)


def turbulence_fields(p: SimParams, dtype=np.float32, seed: int = TURB_SEED, b0=1.0):
    """B = b0 xhat + sum dB_m, E = -v x B, P = 0, evaluated per z-plane."""
    g = Grid.from_params(p, dtype)
    (kb, bamp, phib), (kv, vamp, phiv) = turbulence_modes(seed)
    x = g.coords(0, np.float64)
    y = g.coords(1, np.float64)
    z = g.coords(2, np.float64)
    d0, d1, d2 = g.dims
    out = [np.empty((d2, d1, d0), dtype=dtype) for _ in range(7)]
    Y, X = np.meshgrid(y, x, indexing="ij")
    for kk in range(d2):
        B = np.zeros((3, d1, d0))
        B[0] += b0
        for m in range(len(phib)):
            ph = np.sin(kb[m, 0] * X + kb[m, 1] * Y + kb[m, 2] * z[kk] + phib[m])
            B += bamp[m][:, None, None] * ph
        v = np.zeros((3, d1, d0))
        for m in range(len(phiv)):
            ph = np.sin(kv[m, 0] * X + kv[m, 1] * Y + kv[m, 2] * z[kk] + phiv[m])
            v += vamp[m][:, None, None] * ph
        E = -np.cross(v, B, axis=0)
        for c in range(3):
            out[c][kk] = E[c]
            out[3 + c][kk] = B[c]
        out[6][kk] = 0
    return out


# ---------------------------------------------------------------- pulsar


def pulsar_params(N: int = 64, guard: int = 3, half_size: float = 16.0, radius: float = 3.0,
                  omega: float = 0.05, b0: float = 1.0, pml: int = 8,
                  offset: float = 0.5) -> SimParams:
    """Star at the origin of a non-periodic box with an absorbing layer
    (problem 1, as ``src/main-pulsar3d.cpp`` + ``user_pulsar3d_EZ.hpp``).

    The box is shifted by ``offset`` cells so that no grid point sits at
    r = 0, where the dipole is singular (the reference evaluates it there as
    b0 / TINY, a value that differs between its float and FP64 builds)."""
    p = SimParams()
    p.N = [N, N, N]
    p.guard = [guard] * 3
    d = 2 * half_size / N
    p.lower = [-half_size - offset * d] * 3
    p.size = [2 * half_size] * 3
    p.periodic_boundary = [False, False, False]
    p.pml = [pml] * 3
    p.pmllen = max(1, pml // 2)
    p.sigpml = 0.1
    p.problem = 1
    p.radius = radius
    p.omega = omega
    p.b0 = b0
    p.dt = 0.4 * (2 * half_size / N)
    return p


def _dipole2(x, y, z, p1, p2, p3, phase, tiny):
    """b0-less dipole2 of pulsar_impl.hpp:57-78, float64."""
    c, s = math.cos(phase), math.sin(phase)
    p1t, p2t, p3t = p1 * c - p2 * s, p1 * s + p2 * c, p3
    r2 = x * x + y * y + z * z
    pr = p1t * x + p2t * y + p3t * z
    den = np.sqrt(r2 ** 3) + tiny
    return [(3.0 * q * pr / (r2 + tiny) - pq) / den for q, pq in ((x, p1t), (y, p2t), (z, p3t))]


def pulsar_fields(p: SimParams, dtype=np.float32, yee: bool = False):
    """B = b0 * dipole(p1, p2, p3), E = 0, P = 0 at every point
    (``src/user_pulsar3d_EZ.hpp``; the quadrupole terms are zero unless set).
    With `yee`, each B component at its staggered position
    (``src/user_pulsar3d.hpp``, the staggered solver's initial condition)."""
    tiny = 1e-7 if np.dtype(dtype) == np.float32 else 1e-11

    def fn(Z, Y, X, c):
        if c < 3 or c == 6:
            return np.zeros_like(X)
        return p.b0 * _dipole2(X, Y, Z, p.p1, p.p2, p.p3, 0.0, tiny)[c - 3]
    return [a.copy() for a in _per_component(fn, p, dtype, yee)]


# ------------------------------------------------ 2D log-spherical pulsar


def sph_pulsar_params(nr: int = 64, nth: int = 32, guard: int = 4, r_out: float = 100.0,
                      omega: float = 0.2, b0: float = 1.0, pml: int = 8,
                      cfl: float = 0.3) -> SimParams:
    """Aligned dipole star of radius 1 on x = ln r in [0, ln r_out],
    theta in [0, pi], one z plane (``src/main-pulsar2d-spherical.cpp`` +
    ``src/user_pulsar_sph.hpp``).  guard[1] >= 4 because the reference's axis
    boundary writes three rows beyond theta = pi, which is the first guard
    row.  dt = cfl * d(ln r): the smallest cell is r * d(ln r) at r = 1."""
    p = SimParams()
    p.N = [nr, nth, 1]
    p.guard = [guard, guard, 0]
    p.lower = [0.0, 0.0, 0.0]
    p.size = [math.log(r_out), math.pi, 1.0]
    p.periodic_boundary = [False, False, False]
    p.pml = [pml, 0, 0]
    p.pmllen = max(1, pml)
    p.sigpml = 0.1
    p.problem = 1
    p.radius = 1.0
    p.omega = omega
    p.b0 = b0
    p.dt = cfl * math.log(r_out) / nr
    return p


def sph_pulsar_fields(p: SimParams, dtype=np.float32):
    """B^r = b0 2 cos(th) / r^3 / sqrt(g_11), B^th = b0 sin(th) / r^3 /
    sqrt(g_22), B^phi = 0, E = 0, P = 0 (``src/user_pulsar_sph.hpp``;
    dipole_sph_2d, ``pulsar_impl.hpp:131-139``; g_11 = g_22 = r^2), as arrays
    of shape (1, d1, d0)."""
    g = Grid.from_params(p, dtype)
    tiny = 1e-7 if np.dtype(dtype) == np.float32 else 1e-11
    x = g.coords(0, np.float64)
    th = g.coords(1, np.float64)
    TH, X = np.meshgrid(th, x, indexing="ij")
    r = np.exp(X)
    gs = np.maximum(r, tiny)
    zeros = np.zeros_like(X)
    br = p.b0 * (2.0 * np.cos(TH) / r ** 3) / gs
    bt = p.b0 * (np.sin(TH) / r ** 3) / gs
    arrs = [zeros, zeros, zeros, br, bt, zeros, zeros]
    return [np.asarray(a, dtype=dtype)[None].copy() for a in arrs]


# ---------------------------------------------------- 2D cylindrical pulsar


def cyl_pulsar_params(nR: int = 64, nz: int = 128, guard: int = 3, R_max: float = 16.0,
                      radius: float = 2.0, omega: float = 0.1, b0: float = 1.0, pml: int = 8,
                      cfl: float = 0.4) -> SimParams:
    """Aligned dipole star at the origin of an R-z box, R in [0, R_max],
    z in [-R_max, R_max] (``src/main-pulsar2d-cylindrical.cpp`` +
    ``src/user_pulsar.hpp``); the R = 0 axis is the first interior column.
    The z grid is shifted by half a cell so that no point is at the origin."""
    p = SimParams()
    p.N = [nR, nz, 1]
    p.guard = [guard, guard, 0]
    dz = 2 * R_max / nz
    p.lower = [0.0, -R_max - 0.5 * dz, 0.0]
    p.size = [R_max, 2 * R_max, 1.0]
    p.periodic_boundary = [False, False, False]
    p.pml = [pml, pml, 0]
    p.pmllen = max(1, pml // 2)
    p.sigpml = 0.1
    p.problem = 1
    p.radius = radius
    p.omega = omega
    p.b0 = b0
    p.dt = cfl * min(R_max / nR, dz)
    return p


def cyl_pulsar_fields(p: SimParams, dtype=np.float32):
    """B_R, B_z of a dipole of moment b0 R*^3 along z, E = 0, P = 0
    (``src/user_pulsar.hpp``: dipole_x / dipole_z of ``pulsar_impl.hpp:10-50``
    with alpha = phase = 0), as arrays of shape (1, d1, d0)."""
    g = Grid.from_params(p, dtype)
    tiny = 1e-7 if np.dtype(dtype) == np.float32 else 1e-11
    R = g.coords(0, np.float64)
    z = g.coords(1, np.float64)
    Zz, RR = np.meshgrid(z, R, indexing="ij")
    r = np.sqrt(RR * RR + Zz * Zz)
    r = np.where(np.abs(r) < tiny, tiny, r)
    xn, zn = RR / r, Zz / r
    m = p.b0 * p.radius ** 3
    zeros = np.zeros_like(RR)
    bR = m * (3.0 * xn * zn) / (r ** 3 + tiny)
    bz = m * (3.0 * zn * zn - 1.0) / (r ** 3 + tiny)
    arrs = [zeros, zeros, zeros, bR, bz, zeros, zeros]
    return [np.asarray(a, dtype=dtype)[None].copy() for a in arrs]


# ------------------------------------------------ GR Kerr-Schild Wald field


def wald_params(N: int = 48, guard: int = 3, half_size: float = 6.0, a: float = 0.9,
                pml: int = 6, cfl: float = 0.3) -> SimParams:
    """Kerr black hole of spin a (M = 1) at the centre of [-L, L]^3 in
    Cartesian Kerr-Schild coordinates, absorbing layer at the box faces and
    the reference's inner absorbing region inside 0.7 r_H
    (``src/main-gr.cpp`` + ``src/user_wald2.hpp``).  The grid is shifted by
    half a cell so that no point sits on the ring singularity's axis."""
    p = SimParams()
    p.N = [N, N, N]
    p.guard = [guard] * 3
    d = 2 * half_size / N
    p.lower = [-half_size - 0.5 * d] * 3
    p.size = [2 * half_size] * 3
    p.periodic_boundary = [False, False, False]
    p.pml = [pml] * 3
    p.pmllen = max(1, pml // 2)
    p.sigpml = 0.1
    p.a = a
    p.problem = 0
    p.dt = cfl * d
    return p


def cks_sqrt_gamma(a, x, y, z, tiny):
    """sqrt(gamma) of the Kerr-Schild 3-metric (metric_cks_impl.hpp:17-83), float64."""
    R2 = x * x + y * y + z * z
    r = np.sqrt((R2 - a * a + np.sqrt(np.maximum((R2 - a * a) ** 2 + 4.0 * (a * z) ** 2, tiny)))
                / 2.0)
    return np.sqrt(1.0 + 2.0 * r ** 3 / np.maximum(r ** 4 + a * a * z * z, tiny))


def wald_fields(p: SimParams, dtype=np.float32, yee: bool = False):
    """Uniform asymptotic field along the spin axis: B^z = 1 / sqrt(gamma),
    D = 0, P = 0 (``src/user_wald2.hpp``).  With `yee`, the staggered
    solver's initial condition (``src/user_wald.hpp``): B = curl A / sqrt(gamma)
    with A = (-y/2, x/2, 0) (its vector potential at a = 0) taken at the E
    positions and the staggered curl, each component divided by sqrt(gamma)
    at its own position; D = 0."""
    g = Grid.from_params(p, dtype)
    tiny = 1e-7 if np.dtype(dtype) == np.float32 else 1e-11
    if not yee:
        x, y, z = (g.coords(a, np.float64) for a in range(3))
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        bz = 1.0 / cks_sqrt_gamma(p.a, X, Y, Z, tiny)
        zeros = np.zeros_like(X)
        arrs = [zeros, zeros, zeros, zeros, zeros, bz, zeros]
        return [np.asarray(a, dtype=dtype).copy() for a in arrs]
    A = []
    for c, f in enumerate((lambda X, Y: -0.5 * Y, lambda X, Y: 0.5 * X, lambda X, Y: 0.0 * X)):
        Z, Y, X = _xyz(p, dtype, YEE_STAGGER[c])
        A.append(f(X, Y))
    inv = g.inv_delta
    ext = lambda f, ax: np.concatenate([f, f[tuple(slice(-1, None) if i == 2 - ax else
                                                    slice(None) for i in range(3))]],
                                       axis=2 - ax)
    d = lambda f, ax: np.diff(ext(f, ax), axis=2 - ax)
    curl = [d(A[2], 1) * inv[1] - d(A[1], 2) * inv[2],
            d(A[0], 2) * inv[2] - d(A[2], 0) * inv[0],
            d(A[1], 0) * inv[0] - d(A[0], 1) * inv[1]]
    B = []
    for c in range(3):
        Z, Y, X = _xyz(p, dtype, YEE_STAGGER[3 + c])
        B.append(curl[c] / cks_sqrt_gamma(p.a, X, Y, Z, tiny))
    # the last point of each axis has no forward difference: continue the
    # field from the point before it
    for c in range(3):
        for ax in range(3):
            sl = [slice(None)] * 3
            sl[2 - ax] = slice(-1, None)
            src = [slice(None)] * 3
            src[2 - ax] = slice(-2, -1)
            B[c][tuple(sl)] = B[c][tuple(src)]
    zeros = np.zeros_like(B[0])
    return [np.asarray(a, dtype=dtype).copy() for a in (zeros, zeros, zeros, *B, zeros)]