"""The oracle's quantised SGM (oracle_sgm_u16) on a real cost volume: its winner
agrees with the f32 SGM's within one plane, and its sums respect the 16-bit bound."""
import ctypes as C

import numpy as np

from chiaro_b200 import scenes
from chiaro_b200.abi import fptr
from chiaro_b200.depth import output_shape


def test_oracle_u16_winner_within_one_plane(oracle_lib):
    from oracle import oracle
    sc = scenes.workload("tiny", seed=2)
    (cols, rows, step), (cc, cr, cs) = output_shape(sc.width, sc.height, sc.options)
    D = sc.options.planes + 1
    dbg = oracle.debug_buffers(len(sc.cameras), cc * cr, D, cols * rows)
    oracle.refine_multiview_depth(sc.inputs(), 0, sc.alignments(), sc.options, threads=4, debug=dbg)
    agg = np.zeros(cc * cr * D, np.uint16)
    best = np.zeros(cc * cr, np.uint16)
    oracle_lib.oracle_sgm_u16(fptr(dbg["coarse_costs"]), fptr(dbg["coarse_guidance"]), cc, cr, D,
                              agg.ctypes.data_as(C.POINTER(C.c_uint16)), best.ctypes.data_as(C.POINTER(C.c_uint16)))
    assert agg.max() <= 8 * (4608 + 922)
    f32 = 1 + np.argmin(dbg["regularised"].reshape(-1, D)[:, 1:], axis=1)
    tested = dbg["coarse_tested"] == 1
    diff = np.abs(f32.astype(int) - best.astype(int))[tested]
    assert tested.sum() > 100 and (diff <= 1).mean() >= 0.99
