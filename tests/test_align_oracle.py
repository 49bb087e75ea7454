"""The oracle's align_module restatement (align.rs:281-830): the reference's own
homography test (align.rs:869-893) and the module alignment of a rendered scene."""
import ctypes as C

import numpy as np

from chiaro_b200 import abi, scenes

D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)


def _apply(h, a):
    v = h @ np.array([a[0], a[1], 1.0])
    return v[:2] / v[2]


def test_homography_fit_recovers_a_known_transform(oracle_lib):
    truth = np.array([[1.02, 0.01, 5.0], [-0.015, 0.99, -3.0], [1e-6, -2e-6, 1.0]])
    pairs = []
    for y in range(0, 3000, 250):
        for x in range(0, 4000, 250):
            a = (float(x), float(y))
            pairs.append((a, tuple(_apply(truth, a)), 0.9))
    for i in range(20):  # gross outliers
        a = pairs[i * 7][0]
        pairs.append((a, (a[0] + 80.0, a[1] - 120.0), 0.9))
    points = np.array([[p[0][0], p[0][1], p[1][0], p[1][1]] for p in pairs], np.float64)
    scores = np.array([p[2] for p in pairs], np.float32)
    h = np.zeros(9, np.float64)
    inliers = C.c_size_t()
    residuals = np.zeros(len(pairs), np.float32)
    assert oracle_lib.oracle_fit_homography_ransac(points.ctypes.data_as(D), scores.ctypes.data_as(F), len(pairs),
                                                   1.0, h.ctypes.data_as(D), C.byref(inliers),
                                                   residuals.ctypes.data_as(F)) == 1
    assert inliers.value >= 190
    assert residuals[:inliers.value][inliers.value // 2] < 1e-3
    for a in [(100.0, 100.0), (3900.0, 2900.0)]:
        want, got = _apply(truth, a), _apply(h.reshape(3, 3), a)
        assert abs(got[0] - want[0]) < 1e-3 and abs(got[1] - want[1]) < 1e-3


def align_input(scene, i):
    lum = scene.luminance[i]
    data = np.ascontiguousarray(lum.data, np.float32)
    inp = abi.AlignInputC(luminance=data.ctypes.data_as(F), luma_width=lum.width, luma_height=lum.height,
                          width=scene.width, height=scene.height, has_camera=1, camera=scene.cameras[i].to_c(),
                          nominal_focal_px=float(scene.cameras[i].k[0, 0]))
    return inp, data


def default_options():
    """AlignOptions::default() (align.rs:229-243)."""
    return abi.AlignOptionsC(grid_step=32, patch=32, coarse_radius=12, min_score=0.5, inlier_px=3.0,
                             min_inlier_ratio=0.45, refine=1)


def oracle_align(lib, scene, t, options, seed=None, is_reference=False, no_cameras=False):
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
    err = C.create_string_buffer(128)
    st = lib.oracle_align_module(C.byref(ref), C.byref(tgt), int(is_reference), C.byref(options),
                                 C.byref(seed) if seed is not None else None, C.byref(out), C.byref(gain),
                                 C.byref(report), err)
    return st, points, conf, gain.value, report, err.value.decode()


def test_oracle_aligns_a_rendered_module(oracle_lib):
    sc = scenes.workload("small", seed=2)
    options = default_options()
    st, points, conf, gain, report, _ = oracle_align(oracle_lib, sc, 1, options)
    assert st == 0
    assert report.initialised_from == 2 and report.n_levels >= 1
    assert report.accepted == 1 and report.inlier_ratio > 0.45
    assert 0.25 <= gain <= 4.0
    # the scene's warps are the calibrated infinity mapping: the refinement stays close to it
    calibrated = sc.warps[1]
    both = np.isfinite(points.reshape(-1, 2)).all(1) & np.isfinite(calibrated.points).all(1)
    assert both.mean() > 0.5
    st, points_ref, _, gain_ref, report_ref, _ = oracle_align(oracle_lib, sc, 1, options, is_reference=True)
    assert st == 0 and report_ref.status == 0 and gain_ref == 1.0 and report_ref.coverage == 1.0
