"""GPU parity at the benchmark's full size (five_view: 4160x3120 reference, 4 sources, 128 planes).

The oracle needs minutes for a whole full-size stage, so each stage is checked
on its own, fed with the GPU's upstream outputs (which the previous check
covered), bit for bit:

  * cost volume: bands of coarse rows (one through the middle, one at the top
    edge where patches leave the image and the exact per-tap path runs);
  * SGM, winner-take-all and the three consistency filters: the whole grid;
  * direct pass (with its wide-radius retry): bands of fine rows seeded by the
    GPU's coarse field;
  * per-target decisions: a band of fine rows per target, compared on the rows
    whose consensus and boundary neighbourhoods (two rows either side) lie
    inside the band.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import scenes
from chiaro_b200.abi import dptr, fptr, u8ptr
from chiaro_b200.depth import output_shape, pack_views, refine_multiview_depth

from test_gpu_parity import assert_bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full():
    from oracle import oracle
    scene = scenes.workload("five_view", seed=0)
    opt = scene.options
    inputs, alignments = scene.inputs(), scene.alignments()
    (cols, rows, step), (cc, cr, cs) = output_shape(scene.width, scene.height, opt)
    n = len(inputs)
    dbg = oracle.debug_buffers(n, cc * cr, opt.planes + 1, cols * rows)
    dmap = refine_multiview_depth(inputs, scene.reference_index, alignments, opt, debug=dbg)
    assert dmap is not None
    views, keep = pack_views(scene.inputs(), scene.alignments())
    return dict(scene=scene, opt=opt, o=opt.to_c(), dbg=dbg, views=views, keep=keep, n=n, cols=cols, rows=rows,
                cc=cc, cr=cr, D=opt.planes + 1, lib=oracle.lib(), threads=oracle.threads_default())


def _rows(a, start, stop, width):
    return a[start * width:stop * width]


@pytest.mark.parametrize("where", ["middle", "top"])
def test_cost_volume_band(full, where):
    f, L = full, full["lib"]
    cc, cr, D = f["cc"], f["cr"], f["D"]
    a = cr // 2 - 2 if where == "middle" else 0
    b = a + 4
    N = cc * cr
    scores = np.zeros(N * D, np.float32)
    costs = np.zeros(N * D, np.float32)
    guidance = np.zeros(N, np.float32)
    tested = np.zeros(N, np.uint8)
    assert L.oracle_build_cost_volume(f["views"], f["n"], f["scene"].reference_index, C.byref(f["o"]), a, b,
                                      fptr(scores), fptr(costs), fptr(guidance), u8ptr(tested),
                                      f["threads"]) == 0
    dbg = f["dbg"]
    assert_bits(_rows(dbg["coarse_scores"], a, b, cc * D), _rows(scores, a, b, cc * D), "scores")
    assert_bits(_rows(dbg["coarse_costs"], a, b, cc * D), _rows(costs, a, b, cc * D), "costs")
    assert_bits(_rows(dbg["coarse_guidance"], a, b, cc), _rows(guidance, a, b, cc), "guidance")
    assert_bits(_rows(dbg["coarse_tested"], a, b, cc), _rows(tested, a, b, cc), "tested")


def test_sgm_and_select_whole_grid(full):
    f, L, dbg = full, full["lib"], full["dbg"]
    cc, cr, D, opt = f["cc"], f["cr"], f["D"], f["opt"]
    N = cc * cr
    reg = np.empty(N * D, np.float32)
    L.oracle_semi_global_costs(fptr(dbg["coarse_costs"]), fptr(dbg["coarse_guidance"]), cc, cr, D, fptr(reg))
    assert_bits(dbg["regularised"], reg, "regularised")
    samples = np.empty(opt.planes)
    L.oracle_inverse_depth_samples(opt.near_depth, opt.far_depth, opt.planes, dptr(samples))
    labels = np.ascontiguousarray(np.concatenate([[np.nan], samples[::-1]]))
    out = {k: np.zeros(N, t) for k, t in [("has", np.uint8), ("depth", np.float64), ("confidence", np.float32),
                                          ("improvement", np.float32), ("regularized", np.uint8),
                                          ("fillable", np.uint8)]}
    L.oracle_select_depths(dptr(labels), D, fptr(dbg["coarse_scores"]), fptr(dbg["regularised"]),
                           u8ptr(dbg["coarse_tested"]), N, C.byref(f["o"]), u8ptr(out["has"]), dptr(out["depth"]),
                           fptr(out["confidence"]), fptr(out["improvement"]), u8ptr(out["regularized"]),
                           u8ptr(out["fillable"]))
    if opt.completion_iterations == 0:
        assert_bits(dbg["coarse_has"], out["has"], "coarse has")
        m = out["has"] == 1
        assert m.sum() > N // 4
        for k in ("depth", "confidence", "improvement"):
            assert_bits(dbg["coarse_" + k][m], out[k][m], "coarse " + k)
        assert_bits(dbg["coarse_regularized"], out["regularized"], "coarse regularized")
        assert_bits(dbg["coarse_fillable"], out["fillable"], "coarse fillable")


@pytest.mark.parametrize("where", ["middle", "bottom"])
def test_direct_pass_band(full, where):
    f, L, dbg = full, full["lib"], full["dbg"]
    cols, rows = f["cols"], f["rows"]
    a = rows // 2 - 4 if where == "middle" else rows - 6
    b = min(rows, a + 8)
    M = cols * rows
    out = {k: np.zeros(M, t) for k, t in [("has", np.uint8), ("depth", np.float64), ("confidence", np.float32),
                                          ("improvement", np.float32), ("guidance", np.float32),
                                          ("tested", np.uint8)]}
    assert L.oracle_measure_direct_depths(
        f["views"], f["n"], f["scene"].reference_index, C.byref(f["o"]), u8ptr(dbg["coarse_has"]),
        dptr(dbg["coarse_depth"]), fptr(dbg["coarse_confidence"]), fptr(dbg["coarse_improvement"]),
        u8ptr(dbg["coarse_regularized"]), a, b, u8ptr(out["has"]), dptr(out["depth"]), fptr(out["confidence"]),
        fptr(out["improvement"]), fptr(out["guidance"]), u8ptr(out["tested"]), f["threads"]) == 0
    for k in ("has", "guidance", "tested"):
        assert_bits(_rows(dbg["direct_" + k], a, b, cols), _rows(out[k], a, b, cols), "direct " + k)
    m = _rows(out["has"], a, b, cols) == 1
    assert m.sum() > 0
    for k in ("depth", "confidence", "improvement"):
        assert_bits(_rows(dbg["direct_" + k], a, b, cols)[m], _rows(out[k], a, b, cols)[m], "direct " + k)


def test_filters_whole_grid(full):
    f, L, dbg, opt = full, full["lib"], full["dbg"], full["opt"]
    cols, rows = f["cols"], f["rows"]
    istep = (1.0 / opt.near_depth - 1.0 / opt.far_depth) / (opt.planes - 1)
    has = dbg["direct_has"].copy()
    depth = dbg["direct_depth"].copy()
    conf, guid = dbg["direct_confidence"], dbg["direct_guidance"]
    L.oracle_reject_isolated(u8ptr(has), dptr(depth), fptr(conf), fptr(guid), cols, rows, istep * 2.5)
    assert_bits(dbg["isolated_has"], has, "isolated")
    L.oracle_reject_small_components(u8ptr(has), dptr(depth), fptr(guid), cols, rows, istep * 2.5, 24)
    assert_bits(dbg["component_has"], has, "components")
    L.oracle_fit_local_planes(u8ptr(has), dptr(depth), fptr(conf), fptr(guid), cols, rows, istep * 4.0)
    m = has == 1
    assert_bits(dbg["fitted_depth"][m], depth[m], "fitted depth")


def test_decisions_band(full):
    f, L, dbg = full, full["lib"], full["dbg"]
    cols, rows = f["cols"], f["rows"]
    scene = f["scene"]
    M = cols * rows
    a, b = rows // 2 - 6, rows // 2 + 6
    alignments = scene.alignments()
    checked = 0
    for t in range(f["n"]):
        if t == scene.reference_index or not alignments[t].report.accepted or scene.cameras[t] is None:
            continue
        kinds = np.zeros((b - a) * cols, np.uint8)
        assert L.oracle_target_decisions(f["views"], f["n"], scene.reference_index, t, C.byref(f["o"]),
                                         u8ptr(dbg["component_has"]), dptr(dbg["fitted_depth"]),
                                         fptr(dbg["direct_confidence"]), u8ptr(dbg["direct_regularized"]),
                                         fptr(dbg["direct_guidance"]), a, b, u8ptr(kinds)) == 0
        gpu = dbg["decision_kind"][t * M:(t + 1) * M]
        assert_bits(_rows(gpu, a + 2, b - 2, cols), kinds[2 * cols:(b - a - 2) * cols], f"decision kinds {t}")
        checked += 1
    assert checked == f["n"] - 1


def test_quantised_sgm_whole_grid(full, gpu_ctx):
    """The quantised SGM on the full-size cost volume: bit for bit against the integer
    oracle, and its winner within one plane of the f32 path's on the tested nodes."""
    from test_gpu_sgm_u16 import gpu_u16, oracle_u16
    f, dbg = full, full["dbg"]
    cc, cr, D = f["cc"], f["cr"], f["D"]
    agg_g, best_g = gpu_u16(gpu_ctx, dbg["coarse_costs"], dbg["coarse_guidance"], cc, cr, D)
    agg_o, best_o = oracle_u16(dbg["coarse_costs"], dbg["coarse_guidance"], cc, cr, D)
    assert np.array_equal(agg_g, agg_o) and np.array_equal(best_g, best_o)
    f32 = 1 + np.argmin(dbg["regularised"].reshape(-1, D)[:, 1:], axis=1)
    tested = dbg["coarse_tested"] == 1
    diff = np.abs(f32.astype(int) - best_g.astype(int))[tested]
    assert (diff <= 1).mean() >= 0.995
