"""Host logic of batched loops (no GPU): the tile list."""

import numpy as np
import pytest

from pyop2_b200.batch import TILE_DTYPE, build_tiles


def test_tiles_cover_each_segment_exactly_once():
    rng = np.random.default_rng(7)
    sizes = np.concatenate([[0, 1, 255, 256, 257], rng.integers(0, 5000, size=200)])
    for tile in (128, 256, 1024):
        tiles, first = build_tiles(sizes, tile)
        assert tiles.dtype == TILE_DTYPE
        assert first[0] == 0 and len(first) == len(sizes) + 1
        covered = np.zeros(int(sizes.sum()), dtype=np.int64)
        base = np.concatenate([[0], np.cumsum(sizes)])
        for t in range(int(first[-1])):
            s, f = int(tiles["seg"][t]), int(tiles["first"][t])
            assert first[s] <= t < first[s + 1]
            assert 0 <= f < sizes[s] and f % tile == 0
            lo, hi = base[s] + f, base[s] + min(f + tile, sizes[s])
            covered[lo:hi] += 1
        assert (covered == 1).all()


def test_empty_and_bad_input():
    tiles, first = build_tiles([0, 0], 256)
    assert first.tolist() == [0, 0, 0] and len(tiles) == 1
    with pytest.raises(ValueError):
        build_tiles([-1], 256)
    with pytest.raises(ValueError):
        build_tiles([10], 0)
