"""The quantised SGM (chiaro_sgm_aggregate_u16): bit for bit against the oracle's
integer restatement (oracle_sgm_u16), and its winner within one plane of the f32
path's."""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import scenes
from chiaro_b200.abi import fptr
from chiaro_b200.depth import output_shape

pytestmark = pytest.mark.gpu

U16 = C.POINTER(C.c_uint16)


def oracle_u16(costs, guidance, columns, rows, labels):
    from oracle import oracle
    agg = np.zeros(columns * rows * labels, np.uint16)
    best = np.zeros(columns * rows, np.uint16)
    oracle.lib().oracle_sgm_u16(fptr(costs), fptr(guidance), columns, rows, labels, agg.ctypes.data_as(U16),
                                best.ctypes.data_as(U16))
    return agg, best


def gpu_u16(ctx, costs, guidance, columns, rows, labels):
    agg = np.zeros(columns * rows * labels, np.uint16)
    best = np.zeros(columns * rows, np.uint16)
    ctx.check(ctx.lib.chiaro_sgm_aggregate_u16(ctx.handle, fptr(costs), fptr(guidance), columns, rows, labels,
                                               agg.ctypes.data_as(U16), best.ctypes.data_as(U16)))
    return agg, best


@pytest.mark.parametrize("columns,rows,labels", [(1, 1, 1), (1, 1, 3), (5, 1, 4), (1, 7, 33), (13, 9, 65),
                                                 (40, 31, 97), (31, 40, 129), (17, 23, 193), (9, 5, 256),
                                                 (70, 3, 40), (2, 75, 129), (11, 13, 127), (6, 8, 255)])
def test_u16_sgm_matches_integer_oracle(gpu_ctx, columns, rows, labels):
    rng = np.random.default_rng(columns * 131 + rows * 7 + labels)
    n = columns * rows * labels
    costs = rng.uniform(0, 2.25, n).astype(np.float32)
    costs[rng.random(n) < 0.05] = np.float32(2.25)
    costs[rng.random(n) < 0.01] = np.float32(np.nan)   # quantised as the missing cost
    costs[rng.random(n) < 0.01] = np.float32(7.0)      # clamped to 2.25
    costs[rng.random(n) < 0.01] = np.float32(-0.5)     # clamped to 0
    guidance = rng.uniform(0, 7, columns * rows).astype(np.float32)
    agg_g, best_g = gpu_u16(gpu_ctx, costs, guidance, columns, rows, labels)
    agg_o, best_o = oracle_u16(costs, guidance, columns, rows, labels)
    assert np.array_equal(agg_g, agg_o)
    assert np.array_equal(best_g, best_o)


def test_u16_winner_within_one_plane_of_f32(gpu_ctx):
    from oracle import oracle
    from chiaro_b200.depth import refine_multiview_depth
    sc = scenes.workload("small", seed=7)
    (cols, rows, step), (cc, cr, cs) = output_shape(sc.width, sc.height, sc.options)
    D = sc.options.planes + 1
    dbg = oracle.debug_buffers(len(sc.cameras), cc * cr, D, cols * rows)
    refine_multiview_depth(sc.inputs(), 0, sc.alignments(), sc.options, debug=dbg)
    _, best = gpu_u16(gpu_ctx, dbg["coarse_costs"], dbg["coarse_guidance"], cc, cr, D)
    f32 = 1 + np.argmin(dbg["regularised"].reshape(-1, D)[:, 1:], axis=1)
    tested = dbg["coarse_tested"] == 1
    diff = np.abs(f32.astype(int) - best.astype(int))[tested]
    assert (diff <= 1).mean() >= 0.995 and (diff == 0).mean() >= 0.98


def test_u16_rejects_bad_arguments(gpu_ctx):
    from chiaro_b200 import abi
    x = np.zeros(4, np.float32)
    assert gpu_ctx.lib.chiaro_sgm_aggregate_u16(gpu_ctx.handle, fptr(x), fptr(x), 2, 2, 1, None,
                                                None) == abi.ERR_ARGUMENT
    assert gpu_ctx.lib.chiaro_sgm_aggregate_u16(gpu_ctx.handle, fptr(x), fptr(x), 1, 1, 300, None,
                                                np.zeros(1, np.uint16).ctypes.data_as(U16)) == abi.ERR_ARGUMENT
