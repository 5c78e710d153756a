"""The mixed factorization's whole-region trailing update, checked on the host.

ddlak_mixed_update_grid reports the form and grid of the update of a trailing
region of t tile rows (128 x 128 tiles), and ddlak_mixed_update_cta_tiles decodes
a CTA to the C tiles it writes, with the same functions the tile-pair and
CTA-pair kernels use.  Every lower tile of the region must be written by exactly
one CTA, nothing above the diagonal or past the last tile row; the two CTAs of a
cluster share their tile columns and take consecutive tile rows.  No device work
is involved.
"""
import ctypes
from collections import Counter

import pytest


def _lib():
    from libddla_b200.ddla import _c_api as C
    lib = C.lib
    lib.ddlak_mixed_update_grid.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_longlong)]
    lib.ddlak_mixed_update_grid.restype = ctypes.c_int
    lp = ctypes.POINTER(ctypes.c_longlong)
    lib.ddlak_mixed_update_cta_tiles.argtypes = [ctypes.c_int, ctypes.c_longlong, lp, lp,
                                                 ctypes.POINTER(ctypes.c_int)]
    lib.ddlak_mixed_update_cta_tiles.restype = ctypes.c_int
    return lib


def _grid(lib, t):
    kind, ctas = ctypes.c_int(), ctypes.c_longlong()
    assert lib.ddlak_mixed_update_grid(t, ctypes.byref(kind), ctypes.byref(ctas)) == 0
    return kind.value, ctas.value


@pytest.mark.parametrize("t", list(range(1, 70)) + [127, 128, 129, 255, 256, 257])
def test_update_covers_each_lower_tile_once(t):
    lib = _lib()
    kind, ctas = _grid(lib, t)
    assert kind == (2 if t >= 32 else 1 if t >= 4 else 0)
    if kind == 0:  # single tiles: one CTA per lower tile
        assert ctas == t * (t + 1) // 2
        return
    row, col0, nt = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
    cover = Counter()
    tiles_of = []
    for c in range(ctas):
        assert lib.ddlak_mixed_update_cta_tiles(t, c, ctypes.byref(row), ctypes.byref(col0), ctypes.byref(nt)) == 0
        assert 0 <= nt.value <= 2
        tiles_of.append((row.value, col0.value, nt.value))
        for j in range(col0.value, col0.value + nt.value):
            cover[(row.value, j)] += 1
    assert set(cover) == {(i, j) for i in range(t) for j in range(i + 1)}
    assert set(cover.values()) == {1}
    if kind == 2:
        assert ctas % 2 == 0
        for c in range(0, ctas, 2):
            (r0, c0, _), (r1, c1, _) = tiles_of[c], tiles_of[c + 1]
            assert c0 == c1 and c0 % 2 == 0 and r1 == r0 + 1 and r0 % 2 == 0
    else:
        assert all(n >= 1 for _, _, n in tiles_of)  # every tile-pair CTA writes its first tile


def test_update_grid_argument_errors():
    lib = _lib()
    kind, ctas = ctypes.c_int(), ctypes.c_longlong()
    assert lib.ddlak_mixed_update_grid(0, ctypes.byref(kind), ctypes.byref(ctas)) != 0
    row, col0, nt = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
    args = (ctypes.byref(row), ctypes.byref(col0), ctypes.byref(nt))
    _, n40 = _grid(lib, 40)
    assert lib.ddlak_mixed_update_cta_tiles(40, n40, *args) != 0
    assert lib.ddlak_mixed_update_cta_tiles(40, -1, *args) != 0
    assert lib.ddlak_mixed_update_cta_tiles(3, 0, *args) != 0  # single tiles: no pair decoding
