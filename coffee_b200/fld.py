"""Read and write ``*.fld`` field files (format defined in include/coffee_fld.h).

One 80-byte little-endian header, then ``nfields`` arrays of
``dims[0]*dims[1]*dims[2]`` elements, each in the reference's multi_array
order (x fastest: index ``i + j*d0 + k*d0*d1``; reference
``src/data/multi_array_impl.hpp:81-91``).  In numpy the arrays are returned
as C-ordered ``(d2, d1, d0)`` views, so ``a[k, j, i]`` is cell ``(i, j, k)``.
"""
from __future__ import annotations

import struct
import zlib
from dataclasses import dataclass, field

import numpy as np

MAGIC = b"COFFEEF1"
_HDR = struct.Struct("<8s4i3i3iIIdqq")
assert _HDR.size == 80

FIELD_NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "P")
AUX_NAMES = ("Jx", "Jy", "Jz", "divE", "divB")


@dataclass
class FieldFile:
    """Arrays of one field file plus its header values."""

    arrays: list  # list of np.ndarray, shape (d2, d1, d0)
    dims: tuple  # (d0, d1, d2), guards included
    guard: tuple = (0, 0, 0)
    time: float = 0.0
    step: int = 0
    flags: int = 0
    names: list = field(default_factory=list)

    @property
    def dtype(self):
        return self.arrays[0].dtype


def write_fld(path, arrays, guard=(0, 0, 0), time=0.0, step=0, flags=0, crc=True):
    """Write ``arrays`` (all the same dtype and shape ``(d2, d1, d0)``)."""
    arrays = [np.ascontiguousarray(a) for a in arrays]
    dt = arrays[0].dtype
    if dt not in (np.float32, np.float64):
        raise TypeError(f"unsupported dtype {dt}")
    shape = arrays[0].shape
    for a in arrays:
        if a.dtype != dt or a.shape != shape:
            raise ValueError("all arrays must share dtype and shape")
    d2, d1, d0 = shape
    c = 0
    if crc:
        for a in arrays:
            c = zlib.crc32(a.tobytes(), c)
    hdr = _HDR.pack(MAGIC, 1, dt.itemsize, len(arrays), int(flags), d0, d1, d2,
                    *[int(g) for g in guard], c & 0xFFFFFFFF, 0, float(time), int(step), 0)
    with open(path, "wb") as f:
        f.write(hdr)
        for a in arrays:
            f.write(a.tobytes())


def read_fld(path, check_crc=True) -> FieldFile:
    with open(path, "rb") as f:
        raw = f.read()
    (magic, version, esize, nf, flags, d0, d1, d2, g0, g1, g2, c, _r,
     time, step, _r2) = _HDR.unpack_from(raw, 0)
    if magic != MAGIC or version != 1:
        raise ValueError(f"{path}: not a COFFEEF1 field file")
    dt = {4: np.float32, 8: np.float64}[esize]
    n = d0 * d1 * d2
    body = np.frombuffer(raw, dtype=dt, offset=_HDR.size, count=n * nf)
    if check_crc and c != 0:
        got = 0
        for a in range(nf):
            got = zlib.crc32(body[a * n:(a + 1) * n].tobytes(), got)
        if (got & 0xFFFFFFFF) != c:
            raise ValueError(f"{path}: CRC mismatch")
    arrays = [body[a * n:(a + 1) * n].reshape(d2, d1, d0) for a in range(nf)]
    names = list(FIELD_NAMES + AUX_NAMES)[:nf] if nf <= 12 else []
    return FieldFile(arrays, (d0, d1, d2), (g0, g1, g2), time, step, flags, names)
