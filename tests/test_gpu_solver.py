"""GPU behaviour of the library beyond step parity: guard fill, device
initial conditions, diagnostics, restart, determinism, error paths, and
size-independent properties at the 512^3 benchmark size."""
import os

import numpy as np
import pytest

from coffee_b200 import _lib, problems
from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _periodic_fill_np(a, g):
    a = a.copy()
    for ax, axis in ((0, 2), (1, 1), (2, 0)):  # x, y, z in numpy axis order
        gd = g[ax]
        n = a.shape[axis] - 2 * gd
        idx = [slice(None)] * 3
        src = [slice(None)] * 3
        idx[axis] = slice(0, gd)
        src[axis] = slice(n, n + gd)
        a[tuple(idx)] = a[tuple(src)]
        idx[axis] = slice(n + gd, n + 2 * gd)
        src[axis] = slice(gd, 2 * gd)
        a[tuple(idx)] = a[tuple(src)]
    return a


def test_fill_guards_matches_exchange():
    p = problems.alfven_params(16)
    p.N = [16, 24, 20]
    rng = np.random.default_rng(3)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    arrs = [rng.standard_normal(data.shape).astype(np.float32) for _ in range(7)]
    data.upload(arrs)
    data.fill_guards()
    out = data.download()
    for f in range(7):
        assert np.array_equal(out[f], _periodic_fill_np(arrs[f], p.guard))


def test_init_fourier_matches_host_problem():
    p = problems.turbulence_params(32)
    host = problems.turbulence_fields(p, np.float32)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.init_fourier((1.0, 0.0, 0.0), *problems.turbulence_modes())
    dev = data.download()
    for f in range(7):
        assert np.abs(dev[f].astype(np.float64) - host[f]).max() < 2e-6


def _solver(p, fields, semantics="cpu"):
    env = SimEnvironment(p)
    data = SimData(env, fields[0].dtype)
    data.upload(fields)
    return env, data, FieldSolverEZ(data, env, semantics)


def test_determinism_bitwise():
    p = problems.turbulence_params(48)
    f = problems.turbulence_fields(p, np.float32)
    outs = []
    for _ in range(2):
        env, data, s = _solver(p, f)
        s.step(0.0, 3)
        outs.append(data.download())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_restart_is_bitwise(tmp_path):
    p = problems.pulsar_params(N=32, half_size=8.0, radius=2.0, omega=0.1, pml=6)
    f = problems.pulsar_fields(p, np.float32)
    env, data, s = _solver(p, f)
    s.step(0.0, 6)
    full = data.download()
    env2, data2, s2 = _solver(p, f)
    s2.step(0.0, 3)
    t3 = np.float32(0.0)
    for _ in range(3):
        t3 = np.float32(t3 + np.float32(p.dt))
    path = str(tmp_path / "snap.fld")
    s2.save_snapshot(path, float(t3), 3)
    env3, data3, s3 = _solver(p, [np.zeros_like(a) for a in f])
    t, step = s3.load_snapshot(path)
    assert step == 3 and t == pytest.approx(float(t3))
    s3.step(t, 3)
    for a, b in zip(full, data3.download()):
        assert np.array_equal(a, b)


def test_diagnostics_fp64():
    p = problems.pulsar_params(N=32, half_size=8.0, radius=2.0, pml=4)
    f = problems.pulsar_fields(p, np.float32)
    f[0] = (0.01 * f[4]).astype(np.float32)  # some E
    env, data, s = _solver(p, f)
    g = p.guard[0]
    sl = (slice(g, -g),) * 3
    x = problems.Grid.from_params(p).coords(0, np.float32)[g:-g]
    X = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X[0] ** 2 + X[1] ** 2 + X[2] ** 2, dtype=np.float32)
    lo = np.float32(p.lower[0] + p.pml[0] * (p.size[0] / p.N[0]))
    hi = np.float32(p.lower[0] + p.size[0] - p.pml[0] * (p.size[0] / p.N[0]))
    inside = (r >= p.radius)
    for c in X:
        inside &= (c > lo) & (c < hi)
    eB = sum((f[3 + a][sl].astype(np.float64) ** 2) for a in range(3))
    eE = sum((f[a][sl].astype(np.float64) ** 2) for a in range(3))
    assert s.total_energy("B") == pytest.approx(float(eB[inside].sum()), rel=1e-12)
    assert s.total_energy("E") == pytest.approx(float(eE[inside].sum()), rel=1e-12)
    # max |E|/|B| over the interior
    b2 = np.maximum(eB, 1e-7)
    assert s.diag("max_e_over_b") == pytest.approx(float(np.sqrt(eE / b2).max()), rel=1e-6)


def test_nonfinite_is_reported():
    p = problems.alfven_params(16)
    f = problems.alfven_fields(p, np.float32)
    f[4][5, 6, 7] = np.nan
    env, data, s = _solver(p, f)
    with pytest.raises(_lib.CoffeeError) as e:
        s.check_finite()
    assert e.value.code == -5


def test_bad_solver_arguments():
    p = problems.alfven_params(16)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    with pytest.raises(_lib.CoffeeError):
        FieldSolverEZ(data, env, "cpu").step(0.0, -1)


def test_turbulence512_properties():
    """At the benchmark size (512^3 + 3 guards, FP32): after each step the
    clamps hold (E.B = 0 and |E| <= |B| to rounding), every field is finite,
    the guards are exact periodic images, the run is bitwise deterministic
    across two solvers, and B energy changes by less than 1e-3 over 3 steps
    (force-free turbulence evolves slowly at CFL 0.5)."""
    p = problems.turbulence_params(512)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.init_fourier((1.0, 0.0, 0.0), *problems.turbulence_modes())
    s = FieldSolverEZ(data, env, "cpu")
    eb0 = s.total_energy("B")
    s.step(0.0, 3)
    s.check_finite()
    assert s.diag("max_edotb") < 1e-5
    assert s.diag("max_e_over_b") <= 1.0 + 1e-6
    eb1 = s.total_energy("B")
    assert abs(eb1 - eb0) / eb0 < 1e-3
    out = data.download(("Ex", "By", "P"))
    for a in out:
        assert np.array_equal(a, _periodic_fill_np(a, p.guard))
    s.close()
    data2 = SimData(env, np.float32)
    data2.init_fourier((1.0, 0.0, 0.0), *problems.turbulence_modes())
    s2 = FieldSolverEZ(data2, env, "cpu")
    s2.step(0.0, 3)
    out2 = data2.download(("Ex", "By", "P"))
    for a, b in zip(out, out2):
        assert np.array_equal(a, b)


def test_release_order_does_not_matter():
    """The environment may be destroyed before the fields and solvers made on
    it (as a garbage collector may do): they keep it alive, and no error of
    the releases is left for the next call to report."""
    p = problems.alfven_params(16)
    f = problems.alfven_fields(p, np.float32)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(f)
    s = FieldSolverEZ(data, env, "cpu")
    s.step(0.0, 1)
    env.close()
    s.close()
    data.close()
    p2 = problems.turbulence_params(32)
    env2 = SimEnvironment(p2)
    data2 = SimData(env2, np.float32)
    data2.init_fourier((1.0, 0.0, 0.0), *problems.turbulence_modes())
    s2 = FieldSolverEZ(data2, env2, "cpu")
    s2.step(0.0, 1)
    s2.check_finite()
    s2.close()
    data2.close()
    env2.close()
