"""align_module on the GPU (chiaro_align_module) against the oracle's restatement
(align.rs:281-830): the warp, the photometric gain and every report field bit for
bit, for calibrated modules (one and three pyramid levels), a seeded module, the
no-calibration path, refinement off, the reference itself, and the Python API."""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi, scenes
from chiaro_b200.align import AlignInput, AlignOptions, align_module
from test_align_oracle import align_input, default_options, oracle_align

pytestmark = pytest.mark.gpu

F = C.POINTER(C.c_float)


def gpu_align(ctx, scene, t, options, seed=None, is_reference=False, no_cameras=False):
    ref, keep_r = align_input(scene, scene.reference_index)
    tgt, keep_t = align_input(scene, t)
    if no_cameras:
        ref.has_camera = tgt.has_camera = 0
    columns = -(-scene.width // options.grid_step) + 1
    rows = -(-scene.height // options.grid_step) + 1
    points = np.empty(2 * columns * rows, np.float32)
    conf = np.empty(columns * rows, np.float32)
    out = abi.WarpC(capacity=columns * rows, points=points.ctypes.data_as(F), confidence=conf.ctypes.data_as(F))
    gain = C.c_float()
    report = abi.AlignmentReportC()
    st = ctx.lib.chiaro_align_module(ctx.handle, C.byref(ref), C.byref(tgt), int(is_reference), C.byref(options),
                                     C.byref(seed) if seed is not None else None, C.byref(out), C.byref(gain),
                                     C.byref(report))
    return st, points, conf, gain.value, report


def bits(v):
    return np.array([v], np.float32).view(np.uint32)[0]


def same(g, o):
    st_g, pg, cg, gain_g, rg = g
    st_o, po, co, gain_o, ro, _ = o
    assert st_g == st_o == 0
    assert np.array_equal(pg.view(np.uint32), po.view(np.uint32))
    assert np.array_equal(cg.view(np.uint32), co.view(np.uint32))
    assert bits(gain_g) == bits(gain_o)
    for f in ("initialised_from", "status", "accepted", "inliers", "patches", "n_levels"):
        assert getattr(rg, f) == getattr(ro, f), f
    for f in ("coverage", "residual_median_px", "residual_p90_px", "inlier_ratio"):
        assert bits(getattr(rg, f)) == bits(getattr(ro, f)), f
    assert [bits(v) for v in rg.correction_median_px] == [bits(v) for v in ro.correction_median_px]
    for lg, lo in zip(rg.levels[:rg.n_levels], ro.levels[:ro.n_levels]):
        assert (lg.scale, lg.patches, lg.inliers) == (lo.scale, lo.patches, lo.inliers)
        assert bits(lg.median_residual_px) == bits(lo.median_residual_px)


@pytest.mark.parametrize("name,seed", [("small", 2), ("tiny", 1), ("band", 3)])
def test_calibrated_modules_match_the_oracle(gpu_ctx, oracle_lib, name, seed):
    sc = scenes.workload(name, seed=seed)
    options = default_options()
    for t in range(len(sc.cameras)):
        if t == sc.reference_index:
            continue
        g = gpu_align(gpu_ctx, sc, t, options)
        same(g, oracle_align(oracle_lib, sc, t, options))
        assert g[4].initialised_from == 2  # calibration
    assert g[4].n_levels >= (3 if name == "band" else 1)


def test_seeded_and_uncalibrated_modules_match_the_oracle(gpu_ctx, oracle_lib):
    sc = scenes.workload("small", seed=2)
    options = default_options()
    w = sc.warps[1]
    pts = np.ascontiguousarray(w.points, np.float32)
    cf = np.ascontiguousarray(w.confidence, np.float32)
    seed = abi.WarpC(step=w.step, columns=w.columns, rows=w.rows, points=pts.ctypes.data_as(F),
                     confidence=cf.ctypes.data_as(F), capacity=w.columns * w.rows)
    same(gpu_align(gpu_ctx, sc, 1, options, seed=seed), oracle_align(oracle_lib, sc, 1, options, seed=seed))
    for t in (1, 2):
        g = gpu_align(gpu_ctx, sc, t, options, no_cameras=True)
        same(g, oracle_align(oracle_lib, sc, t, options, no_cameras=True))
        assert g[4].initialised_from == 3


def test_refinement_off_and_the_reference_itself(gpu_ctx, oracle_lib):
    sc = scenes.workload("small", seed=2)
    options = default_options()
    options.refine = 0
    g = gpu_align(gpu_ctx, sc, 1, options)
    same(g, oracle_align(oracle_lib, sc, 1, options))
    assert g[4].status == 2 and g[4].n_levels == 0
    g = gpu_align(gpu_ctx, sc, 1, default_options(), is_reference=True)
    same(g, oracle_align(oracle_lib, sc, 1, default_options(), is_reference=True))
    assert g[4].status == 0 and g[3] == 1.0


def test_python_api_and_short_output(gpu_ctx):
    sc = scenes.workload("band", seed=3)
    inputs = sc.inputs()
    result = align_module(inputs[0], inputs[1], AlignOptions(), context=gpu_ctx)
    assert result.report.status == "refined" and result.report.initialised_from == "calibration"
    assert result.report.accepted and len(result.report.levels) == 3 and 0.25 <= result.gain <= 4.0
    self_result = align_module(inputs[0], inputs[0], context=gpu_ctx)
    assert self_result.report.status == "reference"
    ref, keep_r = align_input(sc, 0)
    tgt, keep_t = align_input(sc, 1)
    points = np.empty(8, np.float32)
    out = abi.WarpC(capacity=4, points=points.ctypes.data_as(F))
    gain = C.c_float()
    report = abi.AlignmentReportC()
    options = default_options()
    st = gpu_ctx.lib.chiaro_align_module(gpu_ctx.handle, C.byref(ref), C.byref(tgt), 0, C.byref(options), None,
                                         C.byref(out), C.byref(gain), C.byref(report))
    assert st == abi.ERR_CAPACITY and (out.step, out.columns, out.rows) == (32, 34, 26)


def test_uncorrelated_module_is_the_references_error(gpu_ctx, oracle_lib):
    """Without cameras a featureless tele target (twice the reference's focal length, so
    the search slides it over the reference) gives the no-calibration search nothing to
    correlate: align_module's Err (align.rs:610-617), as CHIARO_INVALID with the message."""
    from chiaro_b200.align import AlignmentError
    from chiaro_b200.image import Plane
    sc = scenes.workload("small", seed=2)
    ref, keep_r = align_input(sc, 0)
    flat = np.full((sc.luminance[1].height, sc.luminance[1].width), 3.0, np.float32)
    tgt, _ = align_input(sc, 1)
    tgt.luminance = flat.ctypes.data_as(F)
    ref.has_camera = tgt.has_camera = 0
    tgt.nominal_focal_px = 2.0 * ref.nominal_focal_px
    options = default_options()
    columns, rows = -(-sc.width // 32) + 1, -(-sc.height // 32) + 1
    points = np.empty(2 * columns * rows, np.float32)
    out = abi.WarpC(capacity=columns * rows, points=points.ctypes.data_as(F))
    gain, report = C.c_float(), abi.AlignmentReportC()
    st = gpu_ctx.lib.chiaro_align_module(gpu_ctx.handle, C.byref(ref), C.byref(tgt), 0, C.byref(options), None,
                                         C.byref(out), C.byref(gain), C.byref(report))
    message = gpu_ctx.lib.chiaro_depth_last_error(gpu_ctx.handle).decode()
    err = C.create_string_buffer(128)
    st_o = oracle_lib.oracle_align_module(C.byref(ref), C.byref(tgt), 0, C.byref(options), None, C.byref(out),
                                          C.byref(gain), C.byref(report), err)
    assert st == st_o == abi.INVALID and message == err.value.decode() and "correlat" in message
    inputs = sc.inputs()
    inputs[0].camera = inputs[1].camera = None
    inputs[0].nominal_focal_px, inputs[1].nominal_focal_px = ref.nominal_focal_px, 2.0 * ref.nominal_focal_px
    inputs[1].luminance = Plane(inputs[1].luminance.width, inputs[1].luminance.height, flat)
    with pytest.raises(AlignmentError):
        align_module(inputs[0], inputs[1], context=gpu_ctx)


def test_wide_windows_and_invalid_arguments(gpu_ctx, oracle_lib):
    sc = scenes.workload("band", seed=3)
    ref, keep_r = align_input(sc, 0)
    tgt, keep_t = align_input(sc, 1)
    points = np.empty(2 * 34 * 26, np.float32)
    out = abi.WarpC(capacity=34 * 26, points=points.ctypes.data_as(F))
    gain, report = C.c_float(), abi.AlignmentReportC()
    wide = default_options()
    wide.patch = 130  # 130 x 130 windows at the finest level (520 px wide): 67 KiB per warp, allowed
    assert gpu_ctx.lib.chiaro_align_module(gpu_ctx.handle, C.byref(ref), C.byref(tgt), 0, C.byref(wide), None,
                                           C.byref(out), C.byref(gain), C.byref(report)) == abi.OK
    wide_points = points.copy()
    st, po, co, go, ro, _ = oracle_align(oracle_lib, sc, 1, wide)
    assert st == 0 and np.array_equal(wide_points.view(np.uint32), po.view(np.uint32))
    # 240 x 240 windows (225 KiB per warp) exceed what a CTA may hold: they need a level at
    # least 960 px wide (a patch is at most a quarter of its level), so 1000 x 1000 planes
    rng = np.random.default_rng(0)
    large = [rng.uniform(0, 7, (1000, 1000)).astype(np.float32) for _ in range(2)]
    for inp, plane in zip((ref, tgt), large):
        inp.luminance = plane.ctypes.data_as(F)
        inp.luma_width = inp.luma_height = 1000
    big = default_options()
    big.patch = 240
    lib, h = gpu_ctx.lib, gpu_ctx.handle
    assert lib.chiaro_align_module(h, C.byref(ref), C.byref(tgt), 0, C.byref(big), None, C.byref(out),
                                   C.byref(gain), C.byref(report)) == abi.ERR_ARGUMENT
    assert lib.chiaro_align_module(h, None, C.byref(tgt), 0, C.byref(big), None, C.byref(out), C.byref(gain),
                                   C.byref(report)) == abi.ERR_ARGUMENT
    zero = default_options()
    zero.grid_step = 0
    assert lib.chiaro_align_module(h, C.byref(ref), C.byref(tgt), 0, C.byref(zero), None, C.byref(out),
                                   C.byref(gain), C.byref(report)) == abi.ERR_ARGUMENT
