"""Python access to the oracle (test infrastructure only).

Two checkers live here, both CPU-only and never part of the product path:

* ``run_port`` - the C restatement in ffe_oracle.c (liboracle.so), which
  follows the reference's field_solver_EZ::evolve_fields step by step
  (reference src/algorithms/field_solver_EZ.cpp:1007-1073 for the CPU build,
  src/algorithms/field_solver_EZ.cu:656-707 for the GPU build).
* ``run_reference`` - the reference's own CPU build (oracle/_ref, compiled by
  oracle/Makefile from the reference sources), driven through a config.toml
  and a .fld input file.
* ``run_reference_gpu`` - the reference's own GPU build of its flat,
  log-spherical, cylindrical and GR solvers (oracle/_ref/coffee_refgpu_*,
  ``make -C oracle gpuref``), the same way; it needs a GPU.

The numpy restatements of the log-spherical, cylindrical and GR solvers are
in axisym_oracle.py and gr_oracle.py.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

from coffee_b200.config import SimParams
from coffee_b200.fld import read_fld, write_fld

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

SEM_CPU_REF = 0
SEM_GPU_REF = 1


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int * 3), ("guard", ctypes.c_int * 3),
        ("lower", ctypes.c_double * 3), ("size", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3), ("shift_ghost", ctypes.c_int),
        ("dt", ctypes.c_double), ("divB_clean", ctypes.c_int),
        ("ch2", ctypes.c_double), ("tau", ctypes.c_double), ("KOeps", ctypes.c_double),
        ("use_edotb_damping", ctypes.c_int), ("damp_gamma", ctypes.c_double),
        ("clean_ep", ctypes.c_int), ("check_egb", ctypes.c_int),
        ("pml", ctypes.c_int * 3), ("pmllen", ctypes.c_int), ("sigpml", ctypes.c_double),
        ("problem", ctypes.c_int),
        ("radius", ctypes.c_double), ("omega", ctypes.c_double), ("b0", ctypes.c_double),
        ("p1", ctypes.c_double), ("p2", ctypes.c_double), ("p3", ctypes.c_double),
        ("q11", ctypes.c_double), ("q12", ctypes.c_double), ("q13", ctypes.c_double),
        ("q22", ctypes.c_double), ("q23", ctypes.c_double),
        ("q_offset_x", ctypes.c_double), ("q_offset_y", ctypes.c_double),
        ("q_offset_z", ctypes.c_double),
        ("tp_start", ctypes.c_double), ("tp_end", ctypes.c_double),
        ("rpert1", ctypes.c_double), ("rpert2", ctypes.c_double), ("dw0", ctypes.c_double),
        ("nT", ctypes.c_double), ("ph1", ctypes.c_double), ("ph2", ctypes.c_double),
        ("dph", ctypes.c_double), ("theta0", ctypes.c_double), ("drpert", ctypes.c_double),
        ("tp_start1", ctypes.c_double), ("tp_end1", ctypes.c_double),
        ("rpert11", ctypes.c_double), ("rpert21", ctypes.c_double), ("dw1", ctypes.c_double),
        ("nT1", ctypes.c_double), ("ph11", ctypes.c_double), ("ph21", ctypes.c_double),
        ("dph1", ctypes.c_double), ("pert_type", ctypes.c_int),
        ("semantics", ctypes.c_int), ("taper_lanes", ctypes.c_int),
    ]


def to_oracle_params(p: SimParams, semantics: int = SEM_CPU_REF, taper_lanes: int = 16):
    o = OracleParams()
    for i in range(3):
        o.N[i] = p.N[i]
        o.guard[i] = p.guard[i]
        o.lower[i] = p.lower[i]
        o.size[i] = p.size[i]
        o.periodic[i] = int(bool(p.periodic_boundary[i]))
        o.pml[i] = p.pml[i]
    for name, _ in OracleParams._fields_:
        if name in ("N", "guard", "lower", "size", "periodic", "pml", "semantics",
                    "taper_lanes"):
            continue
        v = getattr(p, name)
        setattr(o, name, int(v) if isinstance(v, bool) else v)
    o.semantics = semantics
    o.taper_lanes = taper_lanes
    return o


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle port`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, ct in (("oracle_evolve_f32", ctypes.c_float),
                         ("oracle_evolve_f64", ctypes.c_double)):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(OracleParams), ctypes.POINTER(ctypes.POINTER(ct)),
                           ctypes.POINTER(ctypes.POINTER(ct)), ctypes.POINTER(ctypes.POINTER(ct)),
                           ctypes.c_int, ctypes.c_double]
        _lib = lib
    return _lib


def run_port(p: SimParams, fields, nsteps: int, time0: float = 0.0,
             semantics: int = SEM_CPU_REF, taper_lanes: int | None = None, aux: bool = False,
             diag: list | None = None):
    """Advance copies of ``fields`` (7 arrays, float32 or float64) by ``nsteps``
    with the C restatement.  Returns (fields, aux_arrays_or_None).  ``diag``:
    6 arrays dU_EgtB, dU_Epar, dU_KO, dU_EgtB_cum, dU_Epar_cum, dU_KO_cum,
    updated in place (CPU-build semantics)."""
    lib = _load()
    dt = fields[0].dtype
    if taper_lanes is None:
        taper_lanes = 16 if dt == np.float32 else 8
    arrs = [np.ascontiguousarray(a, dtype=dt).copy() for a in fields]
    ct = ctypes.c_float if dt == np.float32 else ctypes.c_double
    P = ctypes.POINTER(ct)
    ptrs = (P * 7)(*[a.ctypes.data_as(P) for a in arrs])
    auxa = None
    auxp = None
    if aux:
        auxa = [np.zeros_like(arrs[0]) for _ in range(5)]
        auxp = (P * 5)(*[a.ctypes.data_as(P) for a in auxa])
    dgp = None
    if diag is not None:
        for a in diag:
            if a.dtype != dt or not a.flags.c_contiguous:
                raise ValueError("diag arrays must be contiguous and of the fields' dtype")
        dgp = (P * 6)(*[a.ctypes.data_as(P) for a in diag])
    op = to_oracle_params(p, semantics, taper_lanes)
    fn = lib.oracle_evolve_f32 if dt == np.float32 else lib.oracle_evolve_f64
    rc = fn(ctypes.byref(op), ptrs, auxp, dgp, int(nsteps), float(time0))
    if rc != 0:
        raise RuntimeError(f"oracle_evolve failed with {rc}")
    return arrs, auxa


def reference_available(dtype=np.float32) -> bool:
    return os.path.exists(ref_binary(dtype))


def ref_binary(dtype=np.float32) -> str:
    return os.path.join(REF_DIR, "coffee_ref_float" if np.dtype(dtype) == np.float32
                        else "coffee_ref_double")


def run_reference(p: SimParams, fields, nsteps: int, time0: float = 0.0, aux: bool = False,
                  workdir: str | None = None, timeout: float | None = None, diag: bool = False):
    """Run the reference's own CPU build.  Returns (fields, aux_or_None, info);
    with ``diag`` info["diag"] holds the energy-change arrays dU_EgtB,
    dU_Epar, dU_KO, dU_EgtB_cum, dU_Epar_cum, dU_KO_cum (the _cum ones zeroed
    before the first step)."""
    dt = fields[0].dtype
    exe = ref_binary(dt)
    if not os.path.exists(exe):
        raise RuntimeError(f"{exe} missing: run `make -C oracle ref REF=<reference checkout>`")
    own = workdir is None
    wd = tempfile.mkdtemp(prefix="coffee_ref_") if own else workdir
    try:
        cfg = os.path.join(wd, "config.toml")
        p.write_toml(cfg)
        fin = os.path.join(wd, "in.fld")
        fout = os.path.join(wd, "out.fld")
        write_fld(fin, fields, guard=tuple(p.guard), time=time0)
        cmd = [exe, fin, fout, str(int(nsteps))] + (["--aux"] if aux else []) + \
            (["--diag"] if diag else [])
        env = dict(os.environ, COFFEE_ORACLE_CONFIG=cfg)
        r = subprocess.run(cmd, cwd=wd, env=env, capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        ff = read_fld(fout)
        out = [a.copy() for a in ff.arrays[:7]]
        auxa = [a.copy() for a in ff.arrays[7:12]] if aux else None
        if diag:
            k = 12 if aux else 7
            info["diag"] = [a.copy() for a in ff.arrays[k:k + 6]]
        return out, auxa, info
    finally:
        if own:
            for f in os.listdir(wd):
                os.unlink(os.path.join(wd, f))
            os.rmdir(wd)


def refgpu_binary(dtype=np.float32) -> str:
    return os.path.join(REF_DIR, "coffee_refgpu_float" if np.dtype(dtype) == np.float32
                        else "coffee_refgpu_double")


def run_reference_gpu(solver: str, p: SimParams, fields, nsteps: int, time0: float = 0.0,
                      aux: bool = False, timeout: float | None = 600, warmup: int = 0):
    """Run the reference's own GPU build (oracle/ref_harness_gpu) of one of
    its solvers: "ez", "sph", "cyl" or "gr".  Needs a GPU.  Returns
    (fields, aux_or_None, info) like run_reference."""
    exe = refgpu_binary(fields[0].dtype)
    if not os.path.exists(exe):
        raise RuntimeError(f"{exe} missing: run `make -C oracle gpuref REF=<reference checkout>`")
    wd = tempfile.mkdtemp(prefix="coffee_refgpu_")
    try:
        cfg = os.path.join(wd, "config.toml")
        p.write_toml(cfg)
        fin = os.path.join(wd, "in.fld")
        fout = os.path.join(wd, "out.fld")
        write_fld(fin, fields, guard=tuple(p.guard), time=time0)
        cmd = [exe, solver, fin, fout, str(int(nsteps))] + (["--aux"] if aux else [])
        if warmup:
            cmd += ["--warmup", str(int(warmup))]
        env = dict(os.environ, COFFEE_ORACLE_CONFIG=cfg)
        r = subprocess.run(cmd, cwd=wd, env=env, capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference GPU run failed ({r.returncode}): {r.stderr[-2000:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        ff = read_fld(fout)
        out = [a.copy() for a in ff.arrays[:7]]
        auxa = [a.copy() for a in ff.arrays[7:12]] if aux else None
        return out, auxa, info
    finally:
        for f in os.listdir(wd):
            os.unlink(os.path.join(wd, f))
        os.rmdir(wd)


def rel_l2(a, b, interior=None):
    """||a - b|| / ||b|| over the interior slice (tuple of slices) in float64;
    when ||b|| is 0 the absolute norm ||a - b|| is returned."""
    if interior is not None:
        a = a[interior]
        b = b[interior]
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / nb if nb > 0 else d


def interior_slices(p: SimParams):
    g = p.guard
    return tuple(slice(g[a], g[a] + p.N[a]) for a in (2, 1, 0))
