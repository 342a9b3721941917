"""Host-side mirror of the reference's ``Coffee::sim_params`` and its TOML keys.

``SimParams`` has the fields, defaults and meaning of ``sim_params``
(reference ``src/sim_params.h:15-124``).  ``from_toml`` reads the keys that
``parse_config`` reads (``src/sim_params.cpp:7-146``) and ``to_toml`` writes
them back, so one ``config.toml`` drives both the reference build used as the
oracle and this library.  ``Grid`` mirrors ``Coffee::Grid``
(``src/data/grid.h:11-266``) as built by ``sim_environment``
(``src/sim_env_impl.hpp:52-60``) for one rank.
"""
from __future__ import annotations

import math
import tomllib
from dataclasses import dataclass, field, fields

import numpy as np

# problem ids (reference src/sim_params.h:66-69)
PROBLEM_PERIODIC = 0
PROBLEM_PULSAR = 1
PROBLEM_ALFVEN_PULSAR = 2


@dataclass
class SimParams:
    dt: float = 0.01
    max_steps: int = 10000
    data_interval: int = 100
    snapshot_interval: int = 1000
    periodic_boundary: list = field(default_factory=lambda: [False, False, False])
    downsample: int = 1
    slice_x: bool = False
    slice_x_pos: float = 0.0
    slice_y: bool = False
    slice_y_pos: float = 0.0
    slice_z: bool = False
    slice_z_pos: float = 0.0
    slice_xy: bool = False
    slice_interval: int = 100
    downsample_2d: int = 1
    N: list = field(default_factory=lambda: [1, 0, 0])
    guard: list = field(default_factory=lambda: [0, 0, 0])
    lower: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    size: list = field(default_factory=lambda: [1.0, 0.0, 0.0])
    nodes: list = field(default_factory=lambda: [1, 0, 0])
    shift_ghost: int = 0
    kn: list = field(default_factory=lambda: [1, 1, 0])
    a: float = 0.99
    calc_current: bool = True
    clean_ep: bool = True
    check_egb: bool = True
    pml: list = field(default_factory=lambda: [60, 60, 60])
    pmllen: int = 10
    sigpml: float = 0.1
    divB_clean: bool = True
    ch2: float = 1.0
    tau: float = 2.0
    KOeps: float = 0.50
    KO_geometry: bool = True
    use_edotb_damping: bool = True
    damp_gamma: float = 0.2
    problem: int = 0
    radius: float = 10.0
    omega: float = 0.001
    b0: float = 1e3
    p1: float = 0.0
    p2: float = 0.0
    p3: float = 1.0
    q11: float = 0.0
    q12: float = 0.0
    q13: float = 0.0
    q22: float = 0.0
    q23: float = 0.0
    q_offset_x: float = 0.0
    q_offset_y: float = 0.0
    q_offset_z: float = 0.0
    tp_start: float = 0.0
    tp_end: float = 0.5
    rpert1: float = 5.0
    rpert2: float = 10.0
    thp1: float = 0.3
    thp2: float = 0.4
    dw0: float = 0.0
    nT: float = 1.0
    shear: float = 0.0
    ph1: float = 3.0 / 16.0
    ph2: float = 5.0 / 16.0
    dph: float = 1.0 / 64.0
    theta0: float = 0.2
    drpert: float = 0.1
    tp_start1: float = 1.0
    tp_end1: float = 1.5
    rpert11: float = 5.0
    rpert21: float = 10.0
    thp11: float = 0.3
    thp21: float = 0.4
    dw1: float = 0.0
    nT1: float = 1.0
    shear1: float = 0.0
    ph11: float = 3.0 * math.pi / 16.0
    ph21: float = 5.0 * math.pi / 16.0
    dph1: float = math.pi / 64.0
    pert_type: int = 0
    skymap_Nth: int = 256
    skymap_Nph: int = 512

    # keys parse_config does not read (it leaves them at their defaults)
    _NOT_PARSED = ("kn", "skymap_Nth", "skymap_Nph")

    @classmethod
    def from_toml(cls, path_or_text: str, is_text: bool = False) -> "SimParams":
        """Parse like ``parse_config``: every missing key keeps its default."""
        if is_text:
            d = tomllib.loads(path_or_text)
        else:
            with open(path_or_text, "rb") as f:
                d = tomllib.load(f)
        p = cls()
        for f_ in fields(cls):
            if f_.name in cls._NOT_PARSED or f_.name not in d:
                continue
            v = d[f_.name]
            cur = getattr(p, f_.name)
            if isinstance(cur, list):
                if len(v) < 3:
                    raise ValueError(f"config key {f_.name!r} needs 3 entries")
                typ = type(cur[0]) if f_.name != "nodes" else int
                setattr(p, f_.name, [typ(x) for x in v[:3]])
            elif isinstance(cur, bool):
                if not isinstance(v, bool):
                    raise ValueError(f"config key {f_.name!r} must be a boolean")
                setattr(p, f_.name, v)
            else:
                setattr(p, f_.name, type(cur)(v))
        return p

    def to_toml(self) -> str:
        out = []
        for f_ in fields(self):
            if f_.name in self._NOT_PARSED:
                continue
            v = getattr(self, f_.name)
            out.append(f"{f_.name} = {_toml_value(f_.name, v)}")
        return "\n".join(out) + "\n"

    def write_toml(self, path):
        with open(path, "w") as f:
            f.write(self.to_toml())


def _toml_value(name, v):
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return repr(float(v))
    if isinstance(v, list):
        if name == "nodes":  # parse_config reads nodes as an array of doubles
            return "[" + ", ".join(repr(float(x)) for x in v) + "]"
        return "[" + ", ".join(_toml_value(name, x) for x in v) + "]"
    raise TypeError(f"cannot write {name}={v!r}")


@dataclass
class Grid:
    """One-rank ``Coffee::Grid`` built from ``SimParams``."""

    dims: tuple
    guard: tuple
    delta: tuple
    inv_delta: tuple
    lower: tuple
    sizes: tuple

    @classmethod
    def from_params(cls, p: SimParams, dtype=np.float32) -> "Grid":
        ft = np.dtype(dtype).type
        dims = tuple(int(p.N[i]) + 2 * int(p.guard[i]) for i in range(3))
        # delta = size / N and inv_delta = 1 / delta in Scalar arithmetic
        delta = tuple(float(ft(p.size[i]) / ft(p.N[i])) if p.N[i] else 1.0 for i in range(3))
        inv = tuple(float(ft(1.0) / ft(d)) for d in delta)
        return cls(dims, tuple(int(g) for g in p.guard), delta, inv,
                   tuple(float(ft(x)) for x in p.lower), tuple(float(ft(x)) for x in p.size))

    def interior(self):
        return tuple(self.dims[i] - 2 * self.guard[i] for i in range(3))

    def coords(self, axis: int, dtype=np.float64):
        """Vertex coordinates ``lower + delta*(n - guard)`` for n in [0, dims)
        (``Grid::pos`` with stagger bit 1, grid.h:116-134), in ``dtype``."""
        ft = np.dtype(dtype).type
        n = np.arange(self.dims[axis], dtype=dtype)
        return ft(self.lower[axis]) + ft(self.delta[axis]) * (n - ft(self.guard[axis]))
