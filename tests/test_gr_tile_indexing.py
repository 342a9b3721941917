"""CPU model of the index arithmetic of the tiled GR stage
(gr_stage_tile_kernel, coffee_b200/csrc/gr_kernels.cuh): for grids of
several shapes, every copy a CTA issues stays inside the arrays, and every
stencil value an active thread reads from its tile was copied there from
the right grid point.  No GPU: the tables and offsets are recomputed here
with the kernel's own formulas."""
import numpy as np
import pytest

TX, TY, H = 32, 8, 2
SX, SY = TX + 2 * H, TY + 2 * H
SP = SX * SY
NT = TX * TY
NLOAD = -(-SP // NT)


def cta_tables(lo, d, bx, by):
    gx0, gy0 = lo[0] + bx * TX - 2, lo[1] + by * TY - 2
    tables = []
    for tid in range(NT):
        row = []
        for m in range(NLOAD):
            e = tid + m * NT
            r, cl = divmod(e, SX)
            lv = e < SP and gx0 + cl < d[0] and gy0 + r < d[1]
            row.append((lv, e, gy0 + r, gx0 + cl))
        tables.append(row)
    return gx0, gy0, tables


@pytest.mark.parametrize("n,guard,shift", [((40, 40, 40), 3, 0), ((80, 80, 80), 3, 0),
                                           ((70, 37, 150), 3, 0), ((33, 9, 5), 4, 1)])
def test_tile_copies_and_stencil_reads_stay_in_bounds(n, guard, shift):
    d = [x + 2 * guard for x in n]
    lo = [guard - shift] * 3
    hi = [d[a] - guard + shift for a in range(3)]
    kchunk = 64
    gx = -(-(hi[0] - lo[0]) // TX)
    gy = -(-(hi[1] - lo[1]) // TY)
    gz = -(-(hi[2] - lo[2]) // kchunk)
    for bz in range(gz):
        k0 = lo[2] + bz * kchunk
        k1 = min(k0 + kchunk, hi[2])
        kend = k1 + 2
        # planes copied: k0 .. kend - 1; window planes from global k0 - 2 .. k0 + 1
        assert k0 - 2 >= 0 and kend - 1 < d[2]
        for bx in range(gx):
            for by in range(gy):
                gx0, gy0, tables = cta_tables(lo, d, bx, by)
                loaded = {}
                for row in tables:
                    for lv, e, gyy, gxx in row:
                        if lv:
                            assert 0 <= gxx < d[0] and 0 <= gyy < d[1]
                            assert e not in loaded
                            loaded[e] = (gyy, gxx)
                for ty in range(TY):
                    for tx in range(TX):
                        i, j = lo[0] + bx * TX + tx, lo[1] + by * TY + ty
                        if not (i < hi[0] and j < hi[1]):
                            continue
                        own = (ty + 2) * SX + tx + 2
                        for off in (-2, -1, 0, 1, 2):
                            for e, want in ((own + off, (j, i + off)),
                                            (own + off * SX, (j + off, i))):
                                assert 0 <= e < SP
                                assert loaded.get(e) == want, (e, want)
