"""The command-line drivers (coffee_b200.cli): the reference's main loop over
the library.  CPU: argument and problem checks, the loop's event schedule,
the initial conditions of the reference snippets the drivers use.  GPU: a
driver run equals stepping through the API directly, and its outputs and
snapshots read back."""
import math
import os

import numpy as np
import pytest

from coffee_b200 import cli, problems
from coffee_b200.config import SimParams
from coffee_b200.fld import read_fld


def _config(tmp_path, p: SimParams, name="config.toml"):
    path = tmp_path / name
    path.write_text(p.to_toml())
    return str(path)


def _with(p, **kw):
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _wave_params(N=16, steps=6):
    p = problems.alfven_params(N)
    p.max_steps = steps
    p.data_interval = 3
    p.snapshot_interval = 4
    p.downsample = 2
    return p


def test_events_follow_the_reference_loop():
    # outputs and snapshots at multiples of the intervals, step 0 included
    ev = cli.events(10, 4, 5)
    assert ev == [(0, True, True), (4, True, False), (5, False, True), (8, True, False),
                  (10, False, True)]
    # after a restart at step 5 nothing is written at step 5 itself
    assert cli.events(10, 4, 5, start=5, restarted=True) == [(8, True, False), (10, False, True)]


def test_problem_id_is_checked(tmp_path):
    p = _wave_params()
    p.problem = 1
    args = cli.parse_args(["wave", "-c", _config(tmp_path, p)])
    with pytest.raises(ValueError, match="problem 0"):
        cli.plan(args)
    args = cli.parse_args(["pulsar3d", "-c", _config(tmp_path, p), "--steps", "3"])
    d, q = cli.plan(args)
    assert d.kind == cli.FLAT and q.max_steps == 3


def test_wave_initial_condition_is_a_force_free_alfven_wave():
    p = _wave_params(32)
    f = problems.alfven_plane_wave_fields(p, np.float64)
    E, B = np.stack(f[:3]), np.stack(f[3:6])
    assert np.abs((E * B).sum(0)).max() < 1e-15          # E.B = 0
    assert abs(np.abs(E).max() - 0.1) < 1e-3              # amplitude xi0
    # E = -v x B with v along B0 at the wave speed is not required, but the
    # wave vector is (2 * 2 pi, 0, 2 pi): E varies along x and z only
    assert np.allclose(E[2][:, 0, :], E[2][:, 5, :])


def test_staggered_wave_initial_condition_is_divergence_free():
    """The staggered branch of user_alfven.hpp: B = B0 + the staggered curl of
    a vector potential, so the cell-centred div B vanishes to rounding, and B
    matches the collocated wave B0 - xi0 sin(k.x) b / w to O(dx^2)."""
    p = problems.alfven_params(N=24, guard=2)
    f = problems.alfven_plane_wave_fields(p, np.float64, yee=True)
    bx, by, bz = f[3:6]
    inv = 24.0
    div = ((bx[:-1, :-1, 1:] - bx[:-1, :-1, :-1]) + (by[:-1, 1:, :-1] - by[:-1, :-1, :-1]) +
           (bz[1:, :-1, :-1] - bz[:-1, :-1, :-1])) * inv
    assert np.abs(div[:-1, :-1, :-1]).max() < 1e-12
    # B_y at its own position (i + 1/2, j, k + 1/2) against the continuum wave
    k = np.array([4 * math.pi, 0.0, 2 * math.pi])
    Z, Y, X = problems._xyz(p, np.float64, problems.YEE_STAGGER[4])
    w = k[0]
    ref = -0.1 * np.sin(k[0] * X + k[2] * Z) * k[0] / w
    err = np.abs(by - ref)[:-1, :-1, :-1].max()
    assert err < 0.1 * (2 * math.pi / 24) ** 2


def test_emwave_initial_condition_is_transverse():
    p = _wave_params(32)
    p.kn = [1, 2, 0]
    f = problems.emwave_fields(p, np.float64)
    kx, ky = 2 * math.pi * 1 / p.size[0], 2 * math.pi * 2 / p.size[1]
    idx = np.unravel_index(np.argmax(np.abs(f[5])), f[5].shape)  # where sin(k.x) is largest
    ex, ey = f[0][idx] / f[5][idx], f[1][idx] / f[5][idx]
    assert abs(ex * kx + ey * ky) < 1e-12 * (kx + ky)       # e . k = 0
    assert abs(math.hypot(ex, ey) - 1) < 1e-12               # unit polarisation
    assert np.abs(f[5]).max() > 0.99 and np.abs(f[3]).max() == 0


@pytest.mark.gpu
def test_wave_driver_equals_api_stepping(tmp_path):
    from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment

    p = _wave_params(16, steps=6)
    cfg = _config(tmp_path, p)
    out = tmp_path / "out"
    assert cli.main(["wave", "-c", cfg, "-o", str(out)]) == 0
    # the same evolve_fields calls through the API
    env = SimEnvironment(p)
    data = SimData(env, np.float32)
    data.upload(problems.alfven_plane_wave_fields(p, np.float32))
    s = FieldSolverEZ(data, env, "cpu")
    s.step(0.0, 3)
    at3 = data.download()
    g = p.guard
    f3 = read_fld(str(out / "fld.00003.fld"))
    for k in range(7):
        want = at3[k][g[2]:-g[2]:2, g[1]:-g[1]:2, g[0]:-g[0]:2]
        assert np.array_equal(f3.arrays[k], want), k
    assert f3.step == 3
    # snapshots at 0 and 4; energies at the outputs 0, 3, 6
    assert os.path.exists(out / "snapshot.00000.fld") and os.path.exists(out / "snapshot.00004.fld")
    lines = (out / "energy.txt").read_text().split("\n")
    assert [int(l.split()[0]) for l in lines if l] == [0, 3, 6]
    s.close()
    data.close()
    env.close()


@pytest.mark.gpu
def test_restart_from_snapshot_continues_the_run(tmp_path):
    p = _wave_params(16, steps=8)
    p.data_interval = 8
    cfg = _config(tmp_path, p)
    a, b = tmp_path / "a", tmp_path / "b"
    assert cli.main(["wave", "-c", cfg, "-o", str(a)]) == 0
    assert cli.main(["wave", "-c", cfg, "-o", str(b),
                     "--restart", str(a / "snapshot.00004.fld")]) == 0
    fa, fb = read_fld(str(a / "fld.00008.fld")), read_fld(str(b / "fld.00008.fld"))
    for x, y in zip(fa.arrays, fb.arrays):
        assert np.array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("driver,make", [
    ("pulsar3d", lambda: problems.pulsar_params(24)),
    ("gr", lambda: problems.wald_params(16)),
    ("pulsar2d-spherical", lambda: problems.sph_pulsar_params(nr=32, nth=16, guard=4)),
    ("pulsar2d-cylindrical", lambda: problems.cyl_pulsar_params(nR=16, nz=32)),
    ("wave-yee", lambda: _wave_params(16)),
    ("pulsar3d-yee", lambda: problems.pulsar_params(24)),
    ("alfven3d-yee", lambda: _with(problems.pulsar_params(24), problem=2)),
    ("gr-yee", lambda: problems.wald_params(16)),
])
def test_every_driver_runs(tmp_path, driver, make):
    p = make()
    p.max_steps, p.data_interval, p.snapshot_interval = 3, 3, 2
    cfg = _config(tmp_path, p)
    out = tmp_path / "out"
    assert cli.main([driver, "-c", cfg, "-o", str(out)]) == 0
    f = read_fld(str(out / "fld.00003.fld"))
    assert f.step == 3 and all(np.isfinite(a).all() for a in f.arrays)
    assert os.path.exists(out / "snapshot.00002.fld")
