"""Host-side logic that needs no GPU: the library loads and exports its C
ABI, parameter defaults and TOML parsing match the reference's sim_params /
parse_config mirror, the field-file format, and the problem set-ups."""
import ctypes
import os
import re

import numpy as np
import pytest

from coffee_b200 import _lib, problems
from coffee_b200.config import Grid, SimParams
from coffee_b200.fld import read_fld, write_fld

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("coffee_b200.h", "coffee_surrogate.h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        names |= set(re.findall(r"COFFEE_API\s+[\w\s\*]+?\b(coffee_\w+)\s*\(", open(h).read()))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    assert set(names) <= set(_lib.SIGNATURES), "binding misses a declared symbol"


def test_version_string():
    assert b"sm_100a" in _lib.load().coffee_version()


def _cparams():
    cp = _lib.CoffeeParams()
    _lib.load().coffee_params_default(ctypes.byref(cp))
    return cp


def _same(cp, sp: SimParams):
    for name, _ in _lib.CoffeeParams._fields_:
        v = getattr(cp, name)
        w = getattr(sp, name)
        if isinstance(w, list):
            assert list(v) == pytest.approx([float(x) for x in w]), name
        else:
            assert float(v) == pytest.approx(float(w)), name


def test_params_defaults_match_sim_params():
    _same(_cparams(), SimParams())


TOML = """
# a config in the style of the reference's config.toml.example
dt = 0.004
max_steps = 100
N = [64, 32, 16]
guard = [3, 3, 3]
lower = [-1.0, -2, 0.5]
size = [2.0, 4.0, 1.0]
periodic_boundary = [true, false, true]
pml = [0, 4, 0]
pmllen = 3
sigpml = 0.25
KOeps = 0.3
use_edotb_damping = false
problem = 1
radius = 2.5
omega = 0.1
b0 = 1e2
p1 = 0.3
q11 = 0.01
nodes = [1, 1, 1]
unknown_key = 7
"""


def test_toml_parse_matches_mirror():
    cp = _lib.CoffeeParams()
    _lib.check(_lib.load().coffee_params_parse_toml(TOML.encode(), ctypes.byref(cp)))
    sp = SimParams.from_toml(TOML, is_text=True)
    _same(cp, sp)
    assert list(cp.N) == [64, 32, 16]
    assert list(cp.periodic_boundary) == [1, 0, 1]
    assert cp.use_edotb_damping == 0 and cp.b0 == 100.0


def test_toml_roundtrip_through_writer():
    sp = SimParams.from_toml(TOML, is_text=True)
    cp = _lib.CoffeeParams()
    _lib.check(_lib.load().coffee_params_parse_toml(sp.to_toml().encode(), ctypes.byref(cp)))
    _same(cp, sp)


def test_toml_rejects_garbage():
    cp = _lib.CoffeeParams()
    rc = _lib.load().coffee_params_parse_toml(b"dt 0.1\n", ctypes.byref(cp))
    assert rc == -2
    assert b"expected key = value" in _lib.load().coffee_last_error_string()


def test_fld_roundtrip_and_crc(tmp_path):
    rng = np.random.default_rng(1)
    arrs = [rng.standard_normal((5, 6, 7)).astype(np.float32) for _ in range(7)]
    path = str(tmp_path / "a.fld")
    write_fld(path, arrs, guard=(3, 3, 3), time=1.5, step=42)
    ff = read_fld(path)
    assert ff.dims == (7, 6, 5) and ff.guard == (3, 3, 3)
    assert ff.time == 1.5 and ff.step == 42
    for a, b in zip(arrs, ff.arrays):
        assert np.array_equal(a, b)
    raw = bytearray(open(path, "rb").read())
    raw[200] ^= 0xFF
    open(path, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="CRC"):
        read_fld(path)


def test_grid_matches_reference_layout():
    p = problems.alfven_params(16)
    g = Grid.from_params(p)
    assert g.dims == (22, 22, 22)
    x = g.coords(0, np.float32)
    assert x[3] == 0.0 and x[4] == np.float32(1 / 16)  # pos(0, guard, 1) = lower


def test_alfven_initial_condition_is_force_free():
    p = problems.alfven_params(16)
    f = problems.alfven_fields(p, np.float64)
    edotb = f[0] * f[3] + f[1] * f[4] + f[2] * f[5]
    assert np.abs(edotb).max() < 1e-15
    assert np.abs(f[6]).max() == 0


def test_turbulence_spectrum_and_drift():
    (kb, bamp, phib), (kv, vamp, phiv) = problems.turbulence_modes()
    n = np.linalg.norm(kb, axis=1) / (2 * np.pi)
    assert n.min() >= 2 and n.max() <= 8 and len(n) == 32
    # dB_m is normal to k_m (divergence free) and |dB_m| ~ 1/|k_m|
    assert np.abs(np.sum(kb * bamp, axis=1)).max() < 1e-12
    amp = np.linalg.norm(bamp, axis=1)
    assert np.allclose(amp * np.linalg.norm(kb, axis=1), (amp * np.linalg.norm(kb, axis=1))[0])
    assert np.sqrt(0.5 * np.sum(amp ** 2)) == pytest.approx(0.3)
    assert np.linalg.norm(vamp, axis=1).sum() == pytest.approx(0.45)
    p = problems.turbulence_params(32)
    f = problems.turbulence_fields(p, np.float64)
    g = p.guard[0]
    sl = (slice(g, -g),) * 3
    dB = np.stack([f[3][sl] - 1.0, f[4][sl], f[5][sl]])
    assert np.sqrt(np.mean(np.sum(dB ** 2, axis=0))) == pytest.approx(0.3, rel=0.05)
    edotb = f[0] * f[3] + f[1] * f[4] + f[2] * f[5]
    assert np.abs(edotb).max() < 1e-14
    e2 = f[0] ** 2 + f[1] ** 2 + f[2] ** 2
    b2 = f[3] ** 2 + f[4] ** 2 + f[5] ** 2
    assert np.sqrt(e2 / b2).max() < 0.45


def test_env_create_without_gpu_reports_cuda_error():
    lib = _lib.load()
    n = ctypes.c_int(0)
    try:
        cudart = ctypes.CDLL("libcudart.so")
        cudart.cudaGetDeviceCount(ctypes.byref(n))
    except OSError:
        pass
    if n.value > 0:
        pytest.skip("a GPU is present")
    cp = _cparams()
    p = problems.alfven_params(16)
    for a in range(3):
        cp.N[a] = p.N[a]
        cp.guard[a] = 3
        cp.size[a] = 1.0
    h = ctypes.c_void_p()
    rc = lib.coffee_env_create(ctypes.byref(cp), 0, ctypes.byref(h))
    assert rc == -3
    assert b"no CUDA device" in lib.coffee_last_error_string()


def test_env_create_rejects_bad_configs():
    lib = _lib.load()
    cp = _cparams()
    cp.N[0], cp.N[1], cp.N[2] = 16, 16, 16
    # every solver reads one point beyond the box (the EZ solvers check for
    # their three when they are created)
    cp.guard[0], cp.guard[1], cp.guard[2] = 0, 3, 3
    cp.size[1] = cp.size[2] = 1.0
    h = ctypes.c_void_p()
    assert lib.coffee_env_create(ctypes.byref(cp), 0, ctypes.byref(h)) == -2
    assert b"guard" in lib.coffee_last_error_string()


@pytest.mark.parametrize("k,c", [(16, 16), (32, 16), (16, 32), (32, 32), (16, 48), (64, 64)])
def test_weight_gradient_workspace_covers_both_kernels(k, c):
    """The workspace size the library reports holds the mma.sync kernel's
    128 chunk partials and the tcgen05 kernel's per-CTA 128 x k partials
    for two CTAs per SM on up to 192 SMs, over every tap group."""
    need_mma = 128 * k * 27 * c * 4
    cbw = {16: 16, 32: 32, 48: 64, 64: 64}[c]
    groups = -(-27 // (128 // cbw))
    need_tc = max(1, 2 * 192 // groups) * groups * 128 * k * 4
    got = _lib.load().coffee_conv3d_backward_weight_workspace(k, c)
    assert got >= need_mma and got >= need_tc


def test_surrogate_entry_points_reject_bad_sizes_without_a_gpu():
    """Argument checks that come before any device work: too many bias
    channels, unsupported channel counts of the tcgen05 weight gradient."""
    lib = _lib.load()
    fake = ctypes.c_void_p(16)  # never dereferenced: the checks fail first
    rc = lib.coffee_bias_grad(fake, 100, 65, fake, None)
    assert rc == -1 and b"64" in lib.coffee_last_error_string()
    rc = lib.coffee_conv3d_backward_weight_tc(fake, fake, 1, 4, 4, 4, 16, 24, fake, fake, None)
    assert rc == -1 and b"16, 32, 48 or 64" in lib.coffee_last_error_string()
    rc = lib.coffee_conv3d_backward_weight_tc(fake, fake, 1, 4, 4, 4, 48, 16, fake, fake, None)
    assert rc == -1 and b"output channels" in lib.coffee_last_error_string()
