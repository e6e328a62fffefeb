"""The two-step kernel's tile layout (kernels_pair.cu: pair_cols, pair_layout,
pair_tile_at), through gc_pair_layout_tile, which runs the kernel's own code
on the host: every output cell of the grid is stored by exactly one tile, for
the uniform rules and the balanced one (shorter tiles on the edge strips and
the perimeter tile rows), on widths and heights at and around every strip and
tile boundary; strips start on 16-byte boundaries and a tile stores only
columns its strip computes, two columns in from an interior side."""
import ctypes

import numpy as np
import pytest

from comcot_b200 import _lib

WIDTHS = [3, 5, 12, 97, 127, 128, 129, 130, 247, 248, 249, 250, 367, 368, 481, 601, 1201, 2401]
HEIGHTS = [3, 4, 7, 9, 10, 22, 23, 41, 81, 140, 501, 1001, 2001]
TYS = [1, 2, 5, 7, 8, 11, 17, 19, 24, 64]


def _tiles(lib, nx, ny, ty, rule):
    n = lib.gc_pair_layout_tile(nx, ny, ty, rule, -1, None)
    assert n > 0
    out = (ctypes.c_int * 5)()
    res = np.zeros((n, 5), np.int64)
    for lt in range(n):
        assert lib.gc_pair_layout_tile(nx, ny, ty, rule, lt, out) == n
        res[lt] = list(out)
    return res


@pytest.mark.parametrize("rule", [0, 1, 2])
def test_every_cell_stored_by_one_tile(rule):
    lib = _lib.load()
    for nx in WIDTHS:
        for ny in HEIGHTS:
            for ty in TYS:
                t = _tiles(lib, nx, ny, ty, rule)
                cover = np.zeros((ny, nx), np.int32)
                for s, lo, hi, j0, h in t:
                    assert s % 4 == 0, (nx, ny, ty, rule, s)
                    assert h >= 1 and 0 <= j0 < ny, (nx, ny, ty, rule, j0, h)
                    assert s <= lo <= hi <= min(s + 127, nx - 1), (nx, s, lo, hi)
                    if lo > 0:
                        assert lo >= s + 4
                    if hi < nx - 1:
                        assert hi <= s + 123
                    cover[j0:min(j0 + h, ny), lo:hi + 1] += 1
                assert (cover == 1).all(), (nx, ny, ty, rule, int(cover.min()), int(cover.max()))


def test_balanced_layout_shortens_the_boundary_tiles():
    """C2's grid at 19-row tiles: 11-row tiles on the west strip and the
    other strips' first and last tile rows, 9-row tiles on the east strip"""
    lib = _lib.load()
    t = _tiles(lib, 2401, 2001, 19, 2)
    s, h, j0 = t[:, 0], t[:, 4], t[:, 3]
    assert set(h[s == 0]) == {11}
    assert set(h[s == s.max()]) == {9}
    inner = (s > 0) & (s < s.max())
    assert set(h[inner & (j0 == 0)]) == {11}
    assert set(h[inner & (j0 == 2001 - 11)]) == {11}
    assert 19 in set(h[inner])
    assert len(t) == 2331
