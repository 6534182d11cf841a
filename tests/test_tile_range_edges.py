"""Tile ranges from the run edges of the tile sort's last digit pass.

The frame's tile sort (lumen_b200/csrc/sort.cu, onesweep_pass_kernel with a
TileRangeSink) writes the tile ranges of binning.mojo:51-73 in its pass over
the highest varying byte without knowing any key's global predecessor. Each
pass tile (256 * items keys of that pass's input) holds its keys in shared
memory in (digit, input order); key j goes to global position
gbase[digit] + j, so a run of equal ids inside a pass tile covers consecutive
positions. The pass takes an atomic minimum of every run start into the
tile's start and an atomic maximum of every run end + 1 into its end; the
ranges start as (-1, -1) and -1 read as unsigned is the largest value.
tile_ranges_kernel then counts the touched tiles and gives each view the
smallest start among its tiles as its first instance.

This restates that rule in numpy and checks it against the oracle's
tile_ranges (the reference's binning over the sorted keys) on ids in
emission-like order, for one and two varying bytes, several pass-tile sizes,
ragged last pass tiles and batches of views (some empty)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle as O  # noqa: E402

UMAX = np.uint64(0xFFFFFFFF)


def last_pass_ranges(ids_in: np.ndarray, shift: int, tile_keys: int, n_tiles: int):
    """The last digit pass over ids_in (the ids in that pass's input order):
    the sorted ids and the ranges written from the run edges of each pass
    tile."""
    K = ids_in.shape[0]
    d = (ids_in >> np.uint64(shift)) & np.uint64(0xFF)
    idx = np.arange(K)
    # global position of every input key: the stable digit sort
    gpos = np.empty(K, np.int64)
    gpos[np.argsort(d, kind="stable")] = idx
    # shared-memory order inside each pass tile: (digit, input order)
    ptile = idx // tile_keys
    order = np.lexsort((idx, d, ptile))
    sk, st, out = ids_in[order], ptile[order], gpos[order]
    same_tile_prev = np.concatenate([[False], st[1:] == st[:-1]])
    same_tile_next = np.concatenate([st[:-1] == st[1:], [False]])
    first = ~same_tile_prev | np.concatenate([[True], sk[1:] != sk[:-1]])
    last = ~same_tile_next | np.concatenate([sk[:-1] != sk[1:], [True]])
    start = np.full(n_tiles, UMAX, np.uint64)
    end = np.full(n_tiles, -1, np.int64)
    np.minimum.at(start, sk[first].astype(np.int64), out[first].astype(np.uint64))
    np.maximum.at(end, sk[last].astype(np.int64), out[last] + 1)
    sorted_ids = np.empty_like(ids_in)
    sorted_ids[gpos] = ids_in
    ranges = np.stack([np.where(start == UMAX, -1, start.astype(np.int64)), end], axis=1).astype(np.int32)
    return sorted_ids, ranges


def ranges_epilogue(ranges: np.ndarray, tile_begin: np.ndarray):
    """tile_ranges_kernel after the pass: touched tiles and each view's first
    instance (the smallest start among its tiles, -1 when none)."""
    start = ranges[:, 0].astype(np.int64)
    touched = int(np.count_nonzero(start >= 0))
    bounds = np.append(tile_begin, ranges.shape[0])
    first = []
    for v in range(tile_begin.shape[0]):
        s = start[bounds[v]:bounds[v + 1]]
        s = s[s >= 0]
        first.append(int(s.min()) if s.size else -1)
    return touched, first


def emission_ids(rng, tiles_per_view, empty_views, k):
    """Tile ids in emission-like order: splats in depth order, each covering a
    small rectangle of its view's tiles (row by row)."""
    tb = np.concatenate([[0], np.cumsum(tiles_per_view)[:-1]])
    out = []
    total = 0
    live = [v for v in range(len(tiles_per_view)) if v not in empty_views]
    while total < k and live:
        v = live[rng.integers(len(live))]
        tx = int(np.ceil(np.sqrt(tiles_per_view[v])))
        ty = (tiles_per_view[v] + tx - 1) // tx
        x0, y0 = rng.integers(0, tx), rng.integers(0, ty)
        w, h = rng.integers(1, 5), rng.integers(1, 4)
        for y in range(y0, min(y0 + h, ty)):
            for x in range(x0, min(x0 + w, tx)):
                t = y * tx + x
                if t < tiles_per_view[v]:
                    out.append(tb[v] + t)
        total = len(out)
    return np.array(out[:k], np.uint64), tb


@pytest.mark.parametrize("tile_keys", [2048, 4096, 6144])
@pytest.mark.parametrize("views", [(8160,), (300, 40, 1000, 5), (8160,) * 8])
def test_run_edge_ranges_equal_the_binning(tile_keys, views):
    rng = np.random.default_rng(tile_keys + len(views))
    tiles_per_view = np.array(views)
    n_tiles = int(tiles_per_view.sum())
    empty = {1} if len(views) == 4 else set()
    for k in (1, 2, tile_keys - 1, tile_keys, tile_keys + 1, 5 * tile_keys + 17, 150_000):
        ids, tb = emission_ids(rng, tiles_per_view, empty, k)
        if ids.size < 2:
            continue
        # the last pass reads the ids sorted by every lower varying byte
        nbytes = max(1, (int(n_tiles - 1).bit_length() + 7) // 8)
        shift = 8 * (nbytes - 1)
        ids_in = ids[np.argsort(ids & np.uint64((1 << shift) - 1), kind="stable")] if shift else ids
        sorted_ids, ranges = last_pass_ranges(ids_in, shift, tile_keys, n_tiles)
        np.testing.assert_array_equal(sorted_ids, np.sort(ids, kind="stable"))
        ref = O.tile_ranges(sorted_ids << np.uint64(32), n_tiles)
        np.testing.assert_array_equal(ranges, ref)
        touched, first = ranges_epilogue(ranges, tb)
        assert touched == np.unique(ids).size
        for v in range(len(views)):
            in_v = (sorted_ids >= tb[v]) & (sorted_ids < tb[v] + tiles_per_view[v])
            assert first[v] == (int(np.argmax(in_v)) if in_v.any() else -1)
