"""The banded SGM with its full-range fallback (chiaro_sgm_banded), windowed and
over the whole grid: winner labels and fallback tiles identical to the oracle's
restatement (oracle_sgm_banded)."""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import band as bandmod
from chiaro_b200 import scenes
from chiaro_b200.abi import fptr
from chiaro_b200.depth import output_shape

pytestmark = pytest.mark.gpu

I32 = C.POINTER(C.c_int32)
U8 = C.POINTER(C.c_uint8)


def oracle_band(costs, guidance, columns, rows, labels, offsets, tile, band, margin):
    from oracle import oracle
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    winner = np.zeros(columns * rows, np.int32)
    fallback = np.zeros(tx * ty, np.uint8)
    st = oracle.lib().oracle_sgm_banded(fptr(costs), fptr(guidance), columns, rows, labels,
                                        offsets.ctypes.data_as(C.POINTER(C.c_int)), tile, band, margin,
                                        winner.ctypes.data_as(C.POINTER(C.c_int)), fallback.ctypes.data_as(U8))
    assert st == 0
    return winner, fallback


def gpu_band(ctx, costs, guidance, columns, rows, labels, offsets, tile, band, margin):
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    winner = np.zeros(columns * rows, np.int32)
    fallback = np.zeros(tx * ty, np.uint8)
    ctx.check(ctx.lib.chiaro_sgm_banded(ctx.handle, fptr(costs), fptr(guidance), columns, rows, labels,
                                        offsets.ctypes.data_as(I32), tile, band, margin,
                                        winner.ctypes.data_as(I32), fallback.ctypes.data_as(U8)))
    return winner, fallback


@pytest.mark.parametrize("columns,rows,labels,tile,band,margin", [
    (9, 7, 33, 4, 24, 4), (40, 31, 129, 4, 24, 8), (23, 45, 193, 3, 32, 16), (60, 2, 65, 5, 8, 0),
    (1, 30, 40, 1, 1, 2), (17, 17, 97, 2, 16, 6), (64, 48, 97, 4, 31, 1), (50, 40, 65, 4, 24, 200)])
def test_banded_sgm_matches_oracle(gpu_ctx, columns, rows, labels, tile, band, margin):
    rng = np.random.default_rng(columns * 97 + rows * 13 + labels + band)
    n = columns * rows
    costs = rng.uniform(0, 2.25, n * labels).astype(np.float32)
    costs[rng.random(costs.size) < 0.05] = np.float32(2.25)
    guidance = rng.uniform(0, 7, n).astype(np.float32)
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    offsets = rng.integers(1, labels - band + 1, tx * ty).astype(np.int32)  # bands jump freely between tiles
    w_g, f_g = gpu_band(gpu_ctx, costs, guidance, columns, rows, labels, offsets, tile, band, margin)
    w_o, f_o = oracle_band(costs, guidance, columns, rows, labels, offsets, tile, band, margin)
    assert np.array_equal(f_g, f_o)
    assert np.array_equal(w_g, w_o)


def test_banded_sgm_on_a_real_volume(gpu_ctx):
    from oracle import oracle
    from chiaro_b200.depth import refine_multiview_depth
    sc = scenes.workload("small", seed=4, options=dict(planes=192))
    (cols, rows, step), (cc, cr, cs) = output_shape(sc.width, sc.height, sc.options)
    D = sc.options.planes + 1
    dbg = oracle.debug_buffers(len(sc.cameras), cc * cr, D, cols * rows)
    refine_multiview_depth(sc.inputs(), 0, sc.alignments(), sc.options, debug=dbg)
    offsets = bandmod.naive_tile_offsets(dbg["coarse_costs"], cc, cr, D)
    w_g, f_g = gpu_band(gpu_ctx, dbg["coarse_costs"], dbg["coarse_guidance"], cc, cr, D, offsets, 4, 24, 16)
    w_o, f_o = oracle_band(dbg["coarse_costs"], dbg["coarse_guidance"], cc, cr, D, offsets, 4, 24, 16)
    assert np.array_equal(f_g, f_o) and np.array_equal(w_g, w_o)
    assert 0 < f_g.mean() < 1


def test_banded_sgm_refuses_offsets_outside_the_labels(gpu_ctx):
    from chiaro_b200 import abi
    costs = np.zeros(4 * 4 * 33, np.float32)
    guidance = np.zeros(16, np.float32)
    offsets = np.array([0], np.int32)
    winner = np.zeros(16, np.int32)
    fallback = np.zeros(1, np.uint8)
    assert gpu_ctx.lib.chiaro_sgm_banded(gpu_ctx.handle, fptr(costs), fptr(guidance), 4, 4, 33,
                                         offsets.ctypes.data_as(I32), 4, 24, 2, winner.ctypes.data_as(I32),
                                         fallback.ctypes.data_as(U8)) == abi.ERR_ARGUMENT


def test_few_fallback_tiles_take_windows(gpu_ctx):
    """Costs with one clear minimum per node and bands centred on it, except a few tiles
    whose band is far off: only those fall back, through windows of margin nodes (not the
    whole grid), label for label as in the oracle."""
    rng = np.random.default_rng(21)
    columns, rows, labels, tile, band, margin = 57, 43, 97, 4, 24, 3
    r, c = np.divmod(np.arange(columns * rows), columns)
    best = (40 + 10 * np.sin(c / 9.0) + 8 * np.cos(r / 7.0)).astype(int)
    costs = rng.uniform(0.8, 1.6, (columns * rows, labels)).astype(np.float32)
    costs[np.arange(columns * rows), best] = 0.05
    costs = costs.reshape(-1)
    guidance = rng.uniform(0, 7, columns * rows).astype(np.float32)
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    centres = np.array([np.median(best.reshape(rows, columns)[y * tile:(y + 1) * tile, x * tile:(x + 1) * tile])
                        for y in range(ty) for x in range(tx)])
    offsets = bandmod.centred_offsets(centres, labels, band)
    far = rng.choice(tx * ty, 6, replace=False)
    offsets[far] = np.where(offsets[far] > 40, 1, labels - band)
    w_g, f_g = gpu_band(gpu_ctx, costs, guidance, columns, rows, labels, offsets, tile, band, margin)
    windows = C.c_int()
    gpu_ctx.check(gpu_ctx.lib.chiaro_sgm_banded_report(gpu_ctx.handle, C.byref(windows)))
    w_o, f_o = oracle_band(costs, guidance, columns, rows, labels, offsets, tile, band, margin)
    assert np.array_equal(f_g, f_o) and np.array_equal(w_g, w_o)
    assert 0 < f_g.sum() < 20 and windows.value > 1
