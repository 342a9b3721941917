"""coffee_evolve_noalloc, the step loop that allocates no device memory, for
callers whose device memory is owned by their own allocator or pool, or
that cannot take the device synchronisation an allocation may cause.

It is called through the C ABI on device arrays the test owns, twice in a
row (the static scratch keeps the first call's contents), and each result is
compared with coffee_solver_step on the same fields: the two run the same
kernels on the same inputs, so the fields must be equal bit for bit.  The
second call must leave the device's free memory unchanged.  The file is
named to be collected last; it passes alone in a fresh process and after
the other tests."""
import ctypes

import numpy as np
import pytest

from coffee_b200 import _lib, problems
from coffee_b200.solver import FieldSolverEZ, SimData, SimEnvironment, to_coffee_params
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _cudart():
    for name in ("libcudart.so", "libcudart.so.12"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    import glob
    import os

    import torch  # the wheel ships the runtime next to torch's own libraries
    for path in glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia",
                                       "cuda_runtime", "lib", "libcudart.so*")):
        return ctypes.CDLL(path)
    raise OSError("libcudart not found")


def _free_device_bytes():
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    assert _cudart().cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    return free.value


def _sync():
    assert _cudart().cudaDeviceSynchronize() == 0


def _noalloc(lib, params, ptrs, time, nsteps):
    arr = (ctypes.c_void_p * 7)(*ptrs)
    _lib.check(lib.coffee_evolve_noalloc(ctypes.byref(params), _lib.SEM_CPU_REF, arr,
                                         float(time), int(nsteps), None))


def test_noalloc_matches_solver_twice():
    # non-periodic box with a rotating star and absorbing layers, so the
    # second buffer's frozen guards and the start-of-step copy are exercised
    p = problems.pulsar_params(N=32, half_size=8.0, radius=2.0, omega=0.1, b0=1.0, pml=6)
    f = problems.pulsar_fields(p, np.float32)
    dt = np.float32(p.dt)
    t1 = np.float32(np.float32(0.0) + dt)
    t1b = np.float32(t1 + dt)
    t2 = np.float32(t1b + dt)

    # existing entry point: one call of 2 steps, then one call of 1 step
    env = SimEnvironment(p)
    ref_data = SimData(env, np.float32)
    ref_data.upload(f)
    solver = FieldSolverEZ(ref_data, env, "cpu")
    solver.step(0.0, 2)
    ref1 = ref_data.download()
    solver.step(float(t1b), 1)
    ref2 = ref_data.download()

    # the same two calls through coffee_evolve_noalloc on arrays the test owns
    own = SimData(env, np.float32)
    own.upload(f)
    ptrs = [own.dev_ptr(n) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "P")]
    cp = to_coffee_params(p)
    lib = env.lib
    _noalloc(lib, cp, ptrs, 0.0, 2)
    got1 = own.download()
    free0 = _free_device_bytes()
    _noalloc(lib, cp, ptrs, float(t1b), 1)
    _sync()
    free1 = _free_device_bytes()
    got2 = own.download()
    assert t2 > 0
    assert free1 == free0, f"the second call changed free device memory by {free0 - free1} bytes"
    for name, got, ref in (("first call", got1, ref1), ("second call", got2, ref2)):
        for k in range(7):
            err = rel_l2(got[k], ref[k])
            assert np.array_equal(got[k], ref[k]), \
                f"{name}: field {k} differs from coffee_solver_step (rel L2 {err:.2e})"
    solver.close()
    own.close()
    ref_data.close()
    env.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    p = problems.alfven_params(96)
    cp = to_coffee_params(p)
    lib = _lib.load()
    dummy = (ctypes.c_void_p * 7)(*([16] * 7))  # never dereferenced: the size check comes first
    rc = lib.coffee_evolve_noalloc(ctypes.byref(cp), _lib.SEM_CPU_REF, dummy, 0.0, 1, None)
    assert _lib.ERRORS.get(rc) == "COFFEE_E_INVALID"
    assert b"static scratch" in lib.coffee_last_error_string()
