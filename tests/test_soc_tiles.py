"""The SOC tiling the tile kernels run on (clgpu_debug_soc_tiles, host code
only, no GPU): every cone of dim <= 16 lies in exactly one tile, a tile's
cones are consecutive with contiguous rows, and no tile exceeds its cone or
row limit; larger cones and breaks in the rows end a tile."""
import ctypes

import numpy as np
import pytest

from cuclarabel_b200 import _lib

MAX_DIM = 16


def tiles_of(off, dim, max_cones, max_rows):
    L = _lib.load()
    off = np.ascontiguousarray(off, np.int32)
    dim = np.ascontiguousarray(dim, np.int32)
    cap = len(dim) + 1
    out = np.zeros(2 * cap, np.int32)
    nt = L.clgpu_debug_soc_tiles(off.ctypes.data_as(_lib.ip), dim.ctypes.data_as(_lib.ip),
                                 len(dim), max_cones, max_rows, out.ctypes.data_as(_lib.ip),
                                 cap)
    assert nt >= 0
    return [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(nt)]


def check(off, dim, max_cones, max_rows):
    tiles = tiles_of(off, dim, max_cones, max_rows)
    covered = np.zeros(len(dim), int)
    for c0, c1 in tiles:
        assert 0 <= c0 < c1 <= len(dim)
        assert c1 - c0 <= max_cones
        assert sum(dim[c0:c1]) <= max_rows
        for k in range(c0, c1):
            assert 1 <= dim[k] <= MAX_DIM
            covered[k] += 1
            if k > c0:
                assert off[k] == off[k - 1] + dim[k - 1]
    small = (np.asarray(dim) >= 1) & (np.asarray(dim) <= MAX_DIM)
    assert np.array_equal(covered, small.astype(int))
    return tiles


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("shape", [(32, 256), (64, 512), (128, 1024)])
def test_tiles_cover_every_small_cone_once(seed, shape):
    rng = np.random.default_rng(seed)
    dim = rng.choice([1, 2, 3, 5, 8, 10, 16, 17, 40], size=700,
                     p=[.05, .1, .15, .2, .2, .1, .1, .05, .05])
    off = 1000 + np.concatenate([[0], np.cumsum(dim)[:-1]])
    # an instance boundary: rows jump, so a tile must end there
    off[350:] += 7
    tiles = check(off, dim, *shape)
    assert not any(c0 < 350 < c1 for c0, c1 in tiles)


def test_limits_and_arguments():
    dim = np.full(300, 10, np.int32)
    off = np.arange(300, dtype=np.int32) * 10
    tiles = check(off, dim, 128, 1024)
    assert [c1 - c0 for c0, c1 in tiles][:2] == [102, 102]  # row limit: 102 x 10 <= 1024
    tiles = check(off, dim, 32, 256)
    assert all(c1 - c0 <= 25 for c0, c1 in tiles)
    assert tiles_of(off[:0], dim[:0], 32, 256) == []
    L = _lib.load()
    assert L.clgpu_debug_soc_tiles(None, None, 3, 32, 256, None, 0) == -1
    out = (ctypes.c_int * 2)()
    d = (ctypes.c_int * 3)(10, 10, 10)
    o = (ctypes.c_int * 3)(0, 10, 20)
    assert L.clgpu_debug_soc_tiles(o, d, 3, 1, 256, out, 1) == -1  # three tiles, room for one
