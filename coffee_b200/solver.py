"""Python mirror of the reference's objects on the field-update path.

``SimEnvironment``, ``SimData`` and ``FieldSolverEZ`` carry the names and
meaning of ``Coffee::sim_environment`` (reference src/sim_env.h:17-87),
``Coffee::sim_data`` (src/data/sim_data.h:11-24) and
``Coffee::field_solver_EZ`` (src/algorithms/field_solver_EZ.h:6-33).  Each is
a thin owner of a C-ABI handle of libcoffee_b200.so; all computation runs in
the library's CUDA kernels.  Host arrays are numpy arrays of shape
``(dims[2], dims[1], dims[0])`` in the reference layout (x fastest).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .config import SimParams
from ._lib import CoffeeGrid, CoffeeParams, check

FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "P")


def to_coffee_params(p: SimParams) -> CoffeeParams:
    """SimParams -> coffee_params, field by field."""
    lib = _lib.load()
    cp = CoffeeParams()
    lib.coffee_params_default(ctypes.byref(cp))
    for name, ctype in CoffeeParams._fields_:
        if not hasattr(p, name):
            continue
        v = getattr(p, name)
        if isinstance(v, list):
            arr = getattr(cp, name)
            for i in range(3):
                arr[i] = int(v[i]) if isinstance(arr[i], int) else float(v[i])
        elif isinstance(v, bool):
            setattr(cp, name, int(v))
        else:
            setattr(cp, name, v)
    return cp


class SimEnvironment:
    """One rank of ``sim_environment`` on one GPU."""

    def __init__(self, params: SimParams, device: int = 0):
        self.lib = _lib.load()
        self.sim_params = params
        self._cp = to_coffee_params(params)
        h = ctypes.c_void_p()
        check(self.lib.coffee_env_create(ctypes.byref(self._cp), device, ctypes.byref(h)))
        self.handle = h
        g = CoffeeGrid()
        check(self.lib.coffee_env_grid(self.handle, ctypes.byref(g)))
        self._grid = g

    @classmethod
    def from_toml(cls, text: str, device: int = 0) -> "SimEnvironment":
        """Build from config.toml text parsed by the library (parse_config)."""
        lib = _lib.load()
        cp = CoffeeParams()
        check(lib.coffee_params_parse_toml(text.encode(), ctypes.byref(cp)))
        env = cls.__new__(cls)
        env.lib = lib
        env.sim_params = SimParams.from_toml(text, is_text=True)
        env._cp = cp
        h = ctypes.c_void_p()
        check(lib.coffee_env_create(ctypes.byref(cp), device, ctypes.byref(h)))
        env.handle = h
        g = CoffeeGrid()
        check(lib.coffee_env_grid(h, ctypes.byref(g)))
        env._grid = g
        return env

    def grid(self) -> CoffeeGrid:
        return self._grid

    def params(self) -> CoffeeParams:
        return self._cp

    @property
    def dims(self):
        return tuple(self._grid.dims)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.coffee_env_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SimData:
    """Device-resident E, B, P (+ J, divE, divB on request)."""

    def __init__(self, env: SimEnvironment, dtype=np.float32):
        self.env = env
        self.lib = env.lib
        self.dtype = np.dtype(dtype)
        h = ctypes.c_void_p()
        check(self.lib.coffee_fields_create(env.handle, self.dtype.itemsize, ctypes.byref(h)))
        self.handle = h
        d0, d1, d2 = env.dims
        self.shape = (d2, d1, d0)

    def upload(self, arrays):
        """sync_to_device of E, B, P from 7 host arrays."""
        if len(arrays) != 7:
            raise ValueError("need 7 arrays (Ex Ey Ez Bx By Bz P)")
        for fid, a in enumerate(arrays):
            self.upload_field(fid, a)

    def upload_field(self, fid, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        if a.shape != self.shape:
            raise ValueError(f"array shape {a.shape} != grid {self.shape}")
        check(self.lib.coffee_fields_upload(self.handle, int(fid), a.ctypes.data_as(ctypes.c_void_p)))

    def upload_background(self, arrays):
        """sim_data::B0 (3 host arrays), the background field the staggered
        solver subtracts in curl B."""
        if len(arrays) != 3:
            raise ValueError("need 3 arrays (B0x B0y B0z)")
        for fid, a in zip(("B0x", "B0y", "B0z"), arrays):
            self.upload_field(_lib.FIELD_IDS[fid], a)

    def upload_packed(self, buf: np.ndarray):
        """Upload 7 arrays stored back to back in one (pinned or pageable) buffer."""
        check(self.lib.coffee_fields_upload(self.handle, -1, buf.ctypes.data_as(ctypes.c_void_p)))

    def download_packed(self, buf: np.ndarray):
        check(self.lib.coffee_fields_download(self.handle, -1, buf.ctypes.data_as(ctypes.c_void_p)))

    def download(self, names=FIELD_NAMES):
        """sync_to_host; returns a list of arrays."""
        out = []
        for n in names:
            fid = _lib.FIELD_IDS[n] if isinstance(n, str) else int(n)
            a = np.empty(self.shape, dtype=self.dtype)
            check(self.lib.coffee_fields_download(self.handle, fid, a.ctypes.data_as(ctypes.c_void_p)))
            out.append(a)
        return out

    def init_fourier(self, b0, bmodes, vmodes):
        """Device-side problem set-up: B = b0 + sum bamp sin(kb.x + phib),
        E = -v x B with v = sum vamp sin(kv.x + phiv), P = 0."""
        (kb, bamp, phib), (kv, vamp, phiv) = bmodes, vmodes
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (kb, bamp, phib, kv, vamp, phiv)]
        P = ctypes.POINTER(ctypes.c_double)
        b0a = (ctypes.c_double * 3)(*[float(x) for x in b0])
        check(self.lib.coffee_fields_init_fourier(
            self.handle, b0a, len(arrs[2]), arrs[0].ctypes.data_as(P), arrs[1].ctypes.data_as(P),
            arrs[2].ctypes.data_as(P), len(arrs[5]), arrs[3].ctypes.data_as(P),
            arrs[4].ctypes.data_as(P), arrs[5].ctypes.data_as(P)))

    def dev_ptr(self, name) -> int:
        fid = _lib.FIELD_IDS[name] if isinstance(name, str) else int(name)
        p = ctypes.c_void_p()
        check(self.lib.coffee_fields_ptr(self.handle, fid, ctypes.byref(p)))
        return p.value

    def fill_guards(self):
        check(self.lib.coffee_fields_fill_guards(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.coffee_fields_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FieldSolverEZ:
    """``field_solver_EZ(sim_data&, sim_environment&)`` on the GPU."""

    VARIANT = _lib.VARIANT_FLAT

    def __init__(self, data: SimData, env: SimEnvironment, semantics: str = "cpu",
                 stream: int | None = None):
        self.data = data
        self.env = env
        self.lib = env.lib
        sem = {"cpu": _lib.SEM_CPU_REF, "gpu": _lib.SEM_GPU_REF}[semantics]
        h = ctypes.c_void_p()
        check(self.lib.coffee_solver_create(env.handle, data.handle, self.VARIANT, sem,
                                            ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self.handle = h

    def evolve_fields(self, time: float):
        """One full step (5 LSRK stages + KO), as the reference's evolve_fields."""
        check(self.lib.coffee_solver_step(self.handle, float(time), 1))

    def step(self, time: float, nsteps: int):
        check(self.lib.coffee_solver_step(self.handle, float(time), int(nsteps)))

    def set_aux(self, enable: bool):
        check(self.lib.coffee_solver_set_aux(self.handle, int(bool(enable))))

    def set_arithmetic(self, mode: str):
        """'reference' (the default): the CPU semantics compute every
        operation of the reference CPU build in its order and rounding, so an
        FP32 run gives the float build's fields bit for bit (star and
        absorbing boundaries agree to rounding).  'fast': the same algorithm
        regrouped for fewer instructions, equal to rounding."""
        m = {"reference": 0, "fast": 1}[mode]
        check(self.lib.coffee_solver_set_arithmetic(self.handle, m))

    def set_energy_diag(self, enable: bool):
        """Keep the CPU build's energy-change diagnostics dU_EgtB, dU_Epar,
        dU_KO and their _cum sums (SimData.download(_lib.ENERGY_DIAG_NAMES))."""
        check(self.lib.coffee_solver_set_energy_diag(self.handle, int(bool(enable))))

    def set_taper_lanes(self, lanes: int):
        """SIMD width of the CPU build's P-gradient taper offsets (0: by
        precision, 16 for float and 8 for double as in the reference's two
        builds)."""
        check(self.lib.coffee_solver_set_taper_lanes(self.handle, int(lanes)))

    def set_timing(self, enable: bool):
        check(self.lib.coffee_solver_set_timing(self.handle, int(bool(enable))))

    def last_timing(self):
        """Per-kind device milliseconds and launch counts of the last step call."""
        ms = (ctypes.c_double * 3)()
        n = (ctypes.c_int * 3)()
        tot = ctypes.c_double()
        check(self.lib.coffee_solver_last_timing(self.handle, ms, n, ctypes.byref(tot)))
        kinds = ("stage_first", "stage", "ko")
        return {"ms": dict(zip(kinds, list(ms))), "launches": dict(zip(kinds, list(n))),
                "total_ms": tot.value}

    def launches_per_step(self) -> int:
        return int(self.lib.coffee_solver_launches_per_step(self.handle))

    def diag(self, what: str) -> float:
        out = ctypes.c_double()
        check(self.lib.coffee_diag_reduce(self.handle, _lib.DIAG[what], ctypes.byref(out)))
        return out.value

    def total_energy(self, which: str = "B") -> float:
        """field_solver_EZ::total_energy of E or B, accumulated in FP64."""
        return self.diag("energy_" + which)

    def luminosity(self, r: float) -> float:
        """FP64 Poynting luminosity through the sphere |x| = r (flat solver):
        the flux of E x B out of a shell of one grid spacing around r."""
        out = ctypes.c_double()
        check(self.lib.coffee_diag_luminosity(self.handle, float(r), ctypes.byref(out)))
        return out.value

    def check_finite(self):
        check(self.lib.coffee_solver_check_finite(self.handle))

    def save_snapshot(self, path: str, time: float, step: int):
        check(self.lib.coffee_solver_save_snapshot(self.handle, path.encode(), float(time), int(step)))

    def load_snapshot(self, path: str):
        t = ctypes.c_double()
        s = ctypes.c_int64()
        check(self.lib.coffee_solver_load_snapshot(self.handle, path.encode(), ctypes.byref(t),
                                                   ctypes.byref(s)))
        return t.value, s.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.coffee_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_flat(params: SimParams, fields, nsteps: int, time0: float = 0.0, semantics: str = "cpu",
             aux: bool = False, device: int = 0, arithmetic: str = "reference",
             energy_diag: bool = False):
    """Upload ``fields``, advance ``nsteps`` on the GPU, return the 7 fields
    (and J, divE, divB when ``aux``; with ``energy_diag`` the aux list is
    followed by the 6 energy-change arrays dU_EgtB, dU_Epar, dU_KO and their
    _cum sums)."""
    env = SimEnvironment(params, device)
    data = SimData(env, fields[0].dtype)
    data.upload(fields)
    solver = FieldSolverEZ(data, env, semantics)
    if arithmetic != "reference":
        solver.set_arithmetic(arithmetic)
    if aux:
        solver.set_aux(True)
    if energy_diag:
        solver.set_energy_diag(True)
    solver.step(time0, nsteps)
    out = data.download()
    auxa = data.download(("Jx", "Jy", "Jz", "divE", "divB")) if aux else None
    if energy_diag:
        auxa = (auxa or []) + data.download(_lib.ENERGY_DIAG_NAMES)
    solver.close()
    data.close()
    env.close()
    return out, auxa


class FieldSolverEZSpherical(FieldSolverEZ):
    """``field_solver_EZ_spherical(sim_data&, sim_environment&)``
    (src/algorithms/field_solver_EZ_spherical.h:6-32): the 2D log-spherical
    solver, x = ln r, y = theta, one z plane (N[2] = 1, guard[2] = 0).  The
    reference has it only in its GPU build, which it reproduces."""

    VARIANT = _lib.VARIANT_LOGSPH

    def __init__(self, data: SimData, env: SimEnvironment, stream: int | None = None):
        super().__init__(data, env, semantics="gpu", stream=stream)


class FieldSolverEZCylindrical(FieldSolverEZ):
    """``field_solver_EZ_cylindrical(sim_data&, sim_environment&)``
    (src/algorithms/field_solver_EZ_cylindrical.h:6-30): the 2D R-z solver.
    The reference's solver evolves a P of its own; here P is sim_data's P."""

    VARIANT = _lib.VARIANT_CYL

    def __init__(self, data: SimData, env: SimEnvironment, stream: int | None = None):
        super().__init__(data, env, semantics="gpu", stream=stream)


class FieldSolverGrEZ(FieldSolverEZ):
    """``field_solver_gr_EZ(sim_data&, sim_environment&)``
    (src/algorithms/field_solver_gr_EZ.h:6-32): force-free electrodynamics in
    Cartesian Kerr-Schild coordinates around a black hole of spin
    ``params.a``.  sim_data's E holds the displacement D; J / divE / divB
    (set_aux) receive J, div D and div B."""

    VARIANT = _lib.VARIANT_GR

    def __init__(self, data: SimData, env: SimEnvironment, stream: int | None = None):
        super().__init__(data, env, semantics="gpu", stream=stream)


class FieldSolver(FieldSolverEZ):
    """``field_solver(sim_data&, sim_environment&)`` (src/algorithms/field_solver.h:8-35):
    the staggered (Yee) solver, 2nd-order curl, SSP-RK3, the force-free
    current from rho = div E, and E.B = 0 / |E| <= |B| after the substeps
    (src/algorithms/field_solver.cu:690-726).  E and B sit on the staggered
    positions of src/data/sim_data.cpp:19-25; sim_data's B0
    (``SimData.upload_background``) is subtracted in curl B.  The reference
    has it only in its GPU build.  Problem 1 adds the rotating star; the
    reference's solver treats every other problem id as the plain box."""

    VARIANT = _lib.VARIANT_YEE

    def __init__(self, data: SimData, env: SimEnvironment, stream: int | None = None):
        super().__init__(data, env, semantics="gpu", stream=stream)


class FieldSolverGr(FieldSolverEZ):
    """``field_solver_gr(sim_data&, sim_environment&)`` (src/algorithms/field_solver_gr.h:6-29):
    the staggered solver in Cartesian Kerr-Schild coordinates around a hole
    of spin ``params.a`` (evolve_fields_gr, src/algorithms/field_solver_gr.cu:810-861).
    sim_data's E holds D on the E positions; B on the B positions.  The
    reference has it only in its GPU build.  ``step``'s time is not used."""

    VARIANT = _lib.VARIANT_GRYEE

    def __init__(self, data: SimData, env: SimEnvironment, stream: int | None = None):
        super().__init__(data, env, semantics="gpu", stream=stream)


class SphBatch:
    """Independent log-spherical runs advanced together, one kernel launch
    per phase for all of them (``coffee_batch_*``; no counterpart in the
    reference, which runs one grid per process)."""

    def __init__(self, solvers, stream: int | None = None):
        self.solvers = list(solvers)
        self.lib = self.solvers[0].lib
        n = len(self.solvers)
        arr = (ctypes.c_void_p * n)(*[s.handle.value for s in self.solvers])
        h = ctypes.c_void_p()
        check(self.lib.coffee_batch_create(arr, n, ctypes.c_void_p(stream or 0), ctypes.byref(h)))
        self.handle = h
        self.times = np.zeros(n, dtype=np.float64)

    def step(self, nsteps: int):
        """nsteps evolve_fields calls of every run; self.times advances."""
        t = np.ascontiguousarray(self.times, dtype=np.float64)
        check(self.lib.coffee_batch_step(self.handle,
                                         t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         int(nsteps)))
        self.times = t

    def set_persistent(self, on: bool = True):
        """All steps of a ``step`` call in one cooperative launch with
        bounded grid-wide barriers between the phases (bitwise the same
        results); ``step`` then synchronises and raises ``CoffeeError``
        (COFFEE_E_TIMEOUT) if a barrier wait ran out."""
        check(self.lib.coffee_batch_set_persistent(self.handle, int(bool(on))))

    def set_wait_limit(self, limit_ns: int, stall_block: int = -1):
        """Limit of one barrier wait of the persistent mode (ns); stall_block
        >= 0 makes that CTA leave out its first arrival (a test of the
        limit)."""
        check(self.lib.coffee_batch_set_wait_limit(self.handle, int(limit_ns), int(stall_block)))

    def info(self) -> dict:
        """The autotuner's choice: tile shape, run order, first-stage ms."""
        tx, ty, order, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(self.lib.coffee_batch_info(self.handle, ctypes.byref(tx), ctypes.byref(ty),
                                         ctypes.byref(order), ctypes.byref(ms)))
        return {"tile": [tx.value, ty.value], "order": ["given", "largest first"][order.value],
                "first_stage_ms": ms.value}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.coffee_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

