"""FP64 Poynting luminosity (coffee_diag_luminosity): the numpy restatement
against an analytic flux on the CPU, and the library against the
restatement on the GPU."""
import math

import numpy as np
import pytest

from coffee_b200 import _lib, problems
from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment
from oracle import diagnostics


def _swirl_fields(p, dtype=np.float32):
    """E = (-y, x, 0), B = z-hat: S = E x B = (x, y, 0), whose flux through
    the sphere |x| = r is 8 pi r^3 / 3."""
    g = list(p.guard)
    shape = tuple(p.N[a] + 2 * g[a] for a in (2, 1, 0))
    d = [p.size[a] / p.N[a] for a in range(3)]
    x = p.lower[0] + d[0] * (np.arange(shape[2]) - g[0])
    y = p.lower[1] + d[1] * (np.arange(shape[1]) - g[1])
    Y, X = np.meshgrid(y, x, indexing="ij")
    ex = np.broadcast_to(-Y, shape).astype(dtype)
    ey = np.broadcast_to(X, shape).astype(dtype)
    zero = np.zeros(shape, dtype)
    return [ex, ey, zero, zero.copy(), zero.copy(), np.ones(shape, dtype), zero.copy()]


def _box(N=64, half=1.0):
    p = problems.alfven_params(N)
    d = 2 * half / N
    p.lower = [-half + 0.5 * d] * 3  # no point at the origin
    p.size = [2 * half] * 3
    return p


def test_restatement_matches_analytic_flux():
    p = _box(64)
    f = _swirl_fields(p, np.float64)
    for r in (0.4, 0.6, 0.8):
        got = diagnostics.poynting_luminosity(p, f, r)
        want = 8 * math.pi * r ** 3 / 3
        assert abs(got - want) / want < 0.02, (r, got, want)


def test_restatement_uniform_flux_cancels():
    p = _box(48)
    g = list(p.guard)
    shape = tuple(p.N[a] + 2 * g[a] for a in (2, 1, 0))
    zero = np.zeros(shape)
    # E = y-hat, B = z-hat: S = x-hat everywhere, no net flux through a sphere
    f = [zero, np.ones(shape), zero, zero, zero, np.ones(shape), zero]
    r = 0.6
    scale = 4 * math.pi * r * r  # |S| times the sphere's area
    assert abs(diagnostics.poynting_luminosity(p, f, r)) < 0.02 * scale


@pytest.mark.gpu
def test_library_matches_restatement_analytic():
    p = _box(64)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    f = _swirl_fields(p, np.float32)
    data.upload(f)
    s = FieldSolverEZ(data, env, "cpu")
    for r in (0.3, 0.6, 0.9):
        got = s.luminosity(r)
        want = diagnostics.poynting_luminosity(p, f, r)
        assert abs(got - want) <= 1e-9 * abs(want), (r, got, want)
    with pytest.raises(_lib.CoffeeError):
        s.luminosity(0.0)
    s.close()


@pytest.mark.gpu
def test_library_matches_restatement_pulsar():
    """A rotating star after a few steps: the spindown flux through two
    spheres, library against the restatement on the downloaded fields."""
    p = problems.pulsar_params(48, omega=0.2)
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(problems.pulsar_fields(p, np.float32))
    s = FieldSolverEZ(data, env, "gpu")
    s.step(0.0, 20)
    f = data.download()
    for r in (6.0, 9.0):
        got = s.luminosity(r)
        want = diagnostics.poynting_luminosity(p, f, r)
        assert np.isfinite(got)
        assert abs(got - want) <= 1e-9 * max(abs(want), 1e-30), (r, got, want)
    s.close()
