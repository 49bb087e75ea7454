"""The oracle's banded SGM (oracle_sgm_banded): the band-edge rule at the ends of
the label range, fallback through the full-range SGM (whole-grid and windowed),
and the tile targets the band network learns from."""
import ctypes as C

import numpy as np

from chiaro_b200 import band as bandmod
from chiaro_b200.abi import fptr
from chiaro_b200.bandnet import Sample, tile_targets, wide_tile_fraction

I32 = C.POINTER(C.c_int)
U8 = C.POINTER(C.c_uint8)


def _banded(lib, costs, guidance, columns, rows, labels, offsets, tile, band, margin):
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    winner = np.zeros(columns * rows, np.int32)
    fallback = np.zeros(tx * ty, np.uint8)
    st = lib.oracle_sgm_banded(fptr(costs), fptr(guidance), columns, rows, labels,
                               np.ascontiguousarray(offsets, np.int32).ctypes.data_as(I32), tile, band, margin,
                               winner.ctypes.data_as(I32), fallback.ctypes.data_as(U8))
    assert st == 0
    return winner, fallback


def _full_winners(lib, costs, guidance, columns, rows, labels):
    out = np.zeros(columns * rows * labels, np.float32)
    lib.oracle_semi_global_costs(fptr(costs), fptr(guidance), columns, rows, labels, fptr(out))
    return 1 + np.argmin(out.reshape(-1, labels)[:, 1:], axis=1)


def _node_flags(fallback, columns, rows, tile):
    tx, _ = bandmod.tiles_of(columns, rows, tile)
    r, c = np.divmod(np.arange(columns * rows), columns)
    return fallback[(r // tile) * tx + c // tile].astype(bool)


def test_flat_costs_fall_back_only_away_from_label_one(oracle_lib):
    columns, rows, labels, tile, band = 10, 9, 40, 4, 8
    costs = np.full(columns * rows * labels, 2.25, np.float32)
    guidance = np.zeros(columns * rows, np.float32)
    tiles = np.prod(bandmod.tiles_of(columns, rows, tile))
    w, f = _banded(oracle_lib, costs, guidance, columns, rows, labels, np.ones(tiles), tile, band, 2)
    assert not f.any() and (w == 1).all()  # slot 0 is label 1, the range's own end
    w, f = _banded(oracle_lib, costs, guidance, columns, rows, labels, np.full(tiles, 5), tile, band, 2)
    assert f.all() and (w == 1).all()  # the fallback finds label 1 below the band


def test_top_edge_at_the_last_label_is_not_a_band_edge(oracle_lib):
    columns, rows, labels, tile, band = 8, 8, 30, 4, 6
    costs = np.full((columns * rows, labels), 2.0, np.float32)
    costs[:, labels - 1] = 0.1  # every node's best label is the last one
    costs = costs.reshape(-1)
    guidance = np.zeros(columns * rows, np.float32)
    tiles = np.prod(bandmod.tiles_of(columns, rows, tile))
    w, f = _banded(oracle_lib, costs, guidance, columns, rows, labels, np.full(tiles, labels - band), tile, band, 1)
    assert not f.any() and (w == labels - 1).all()
    w, f = _banded(oracle_lib, costs, guidance, columns, rows, labels, np.full(tiles, labels - band - 1), tile, band,
                   1)
    assert f.all() and (w == labels - 1).all()


def test_all_tiles_falling_back_is_the_full_range_sgm(oracle_lib):
    rng = np.random.default_rng(3)
    columns, rows, labels, tile, band = 23, 17, 50, 4, 6
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    offsets = np.full(tx * ty, 11, np.int32)
    costs = rng.uniform(0, 2.25, (rows, columns, labels)).astype(np.float32)
    costs[:, :, 11:11 + band] = 2.25  # flat inside the (unshifting) band: slot 0 wins at every node
    costs = costs.reshape(-1)
    guidance = rng.uniform(0, 7, columns * rows).astype(np.float32)
    w, f = _banded(oracle_lib, costs, guidance, columns, rows, labels, offsets, tile, band, 0)
    assert f.all()
    # the windows cover the grid: one full-range SGM over the whole grid decides every node
    assert np.array_equal(w, _full_winners(oracle_lib, costs, guidance, columns, rows, labels))


def test_whole_grid_fallback_replaces_only_fallback_tiles(oracle_lib):
    rng = np.random.default_rng(8)
    columns, rows, labels, tile, band = 30, 22, 64, 4, 12
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    costs = rng.uniform(0, 2.25, columns * rows * labels).astype(np.float32)
    guidance = rng.uniform(0, 7, columns * rows).astype(np.float32)
    offsets = rng.integers(1, labels - band + 1, tx * ty).astype(np.int32)
    w0, f0 = _banded(oracle_lib, costs, guidance, columns, rows, labels, offsets, tile, band, 0)
    wbig, fbig = _banded(oracle_lib, costs, guidance, columns, rows, labels, offsets, tile, band, 100)
    assert np.array_equal(f0, fbig) and 0 < f0.sum() < f0.size
    flagged = _node_flags(f0, columns, rows, tile)
    # tiles that kept their band keep their banded winners, whatever the fallback does
    assert np.array_equal(w0[~flagged], wbig[~flagged])
    # a margin past the grid makes every window the whole grid: the full-range SGM's winners
    full = _full_winners(oracle_lib, costs, guidance, columns, rows, labels)
    assert np.array_equal(wbig[flagged], full[flagged])


def test_tile_targets_centre_each_tile_on_its_winner_range():
    columns, rows, labels, tile = 6, 5, 100, 4
    winners = np.full(columns * rows, 50, np.int32)
    winners[0], winners[1] = 20, 40  # tile (0, 0): range 20..50
    mask = np.ones(columns * rows, np.uint8)
    mask[[4, 5, 10, 11, 16, 17, 22, 23, 28, 29]] = 0  # no tested node in the tiles of columns 4-5
    s = Sample(np.zeros(columns * rows * labels, np.float32), np.zeros(columns * rows, np.float32), winners, mask,
               columns, rows, labels)
    t = tile_targets(s, tile, kind="midrange")
    grid = t.winners.reshape(rows, columns)
    assert (grid[:4, :4] == 35).all()  # (20 + 50) / 2
    assert (grid[:4, 4:] == 1).all()  # no tested node: the range's end
    assert (grid[4, :4] == 50).all() and (grid[4, 4:] == 1).all()
    assert t.mask.all()


def test_median_tile_targets_and_wide_tiles():
    columns, rows, labels, tile = 8, 4, 100, 4
    winners = np.full(columns * rows, 50, np.int32).reshape(rows, columns)
    winners[0, :3] = [10, 12, 90]  # tile 0: median 50, span 80
    winners[:, 4:] = 30
    winners[3, 7] = 50  # tile 1: median 30, span 20
    s = Sample(np.zeros(columns * rows * labels, np.float32), np.zeros(columns * rows, np.float32),
               winners.reshape(-1), np.ones(columns * rows, np.uint8), columns, rows, labels)
    t = tile_targets(s, tile).winners.reshape(rows, columns)
    assert (t[:, :4] == 50).all() and (t[:, 4:] == 30).all()
    assert wide_tile_fraction(s, tile, band=24) == 0.5  # span 80 > 21; span 20 fits
