"""Known-answer tests of the reference, ported.

Each test restates one of the reference's own unit tests for the depth path
(crates/chiaro-fusion/src/depth.rs:1897-2171, align.rs:895-905,
geometry.rs:367-393, math.rs:141-160) and runs it against the CPU oracle and,
where the operator exists on the device, against the CUDA library too. These
pin the oracle: it must reproduce every known answer the reference's tests
hold before it may serve as the GPU path's checker.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi
from chiaro_b200.abi import CameraC, DepthMapC, WarpC, dptr, fptr, sizeptr, u8ptr, u16ptr
from chiaro_b200.depth import DenseDepthMap, DepthOptions
from chiaro_b200.align import Warp
from chiaro_b200.camera import IDENTITY, PolynomialDistortion, ResolvedCamera, determinant, inverse
from chiaro_b200.camera import rotation_about_axis

from backends import GpuBackend, OracleBackend

NaN = float("nan")


@pytest.fixture(params=["oracle", pytest.param("gpu", marks=pytest.mark.gpu)])
def backend(request):
    if request.param == "oracle":
        return OracleBackend()
    ctx = request.getfixturevalue("gpu_ctx")
    return GpuBackend(ctx)


# depth.rs:1898-1904
def test_inverse_depth_planes_include_bounds_and_favour_near_resolution(oracle_lib):
    out = np.empty(5)
    oracle_lib.oracle_inverse_depth_samples(500.0, 100_000.0, 5, dptr(out))
    assert abs(out[0] - 500.0) < 1e-9
    assert abs(out[4] - 100_000.0) < 1e-6
    assert np.all(out[:-1] < out[1:])
    assert out[1] - out[0] < out[4] - out[3]


# depth.rs:1907-1912
def test_sublabel_fit_refines_inverse_depth_between_planes(oracle_lib):
    labels = np.array([NaN, 10_000.0, 5_000.0, 10_000.0 / 3.0])
    costs = np.array([9.0, 2.0, 0.0, 1.0], dtype=np.float32)
    depth = oracle_lib.oracle_sublabel_depth(dptr(labels), 4, fptr(costs), 2)
    assert depth < 5_000.0
    assert depth > 10_000.0 / 3.0


# depth.rs:1915-1921
def test_aggregation_requires_independent_view_support(oracle_lib):
    opt = DepthOptions().to_c()
    out = C.c_float()
    one = np.array([0.9], dtype=np.float32)
    assert oracle_lib.oracle_aggregate(fptr(one), 1, C.byref(opt), C.byref(out)) == 0
    two = np.array([0.9, 0.7], dtype=np.float32)
    assert oracle_lib.oracle_aggregate(fptr(two), 2, C.byref(opt), C.byref(out)) == 1
    assert abs(out.value - 0.8) < 1e-6


# depth.rs:1924-1941
def test_semi_global_matching_completes_an_ambiguous_middle_node(backend):
    labels, columns, rows = 4, 5, 1
    costs = np.ones(columns * labels, dtype=np.float32)
    for column in [0, 1, 3, 4]:
        costs[column * labels + 2] = 0.0
    guidance = np.full(columns, 0.5, dtype=np.float32)
    regularised = backend.sgm(costs, guidance, columns, rows, labels)
    middle = regularised[2 * labels: 3 * labels]
    assert int(np.argmin(middle)) == 2


# depth.rs:1944-1953
def test_diagonal_paths_visit_every_node_in_both_families(oracle_lib):
    for mirrored in (0, 1):
        idx = np.zeros(20, dtype=np.uintp)
        lengths = np.zeros(8, dtype=np.uintp)
        n = oracle_lib.oracle_diagonal_paths(5, 4, mirrored, sizeptr(idx), sizeptr(lengths))
        assert n == 5 + 4 - 1
        assert lengths[:n].sum() == 20
        visits = np.bincount(idx.astype(np.int64), minlength=20)
        assert np.all(visits == 1)


def _refined(dx):
    return (abi.NW_REFINED, (10.0, 20.0), (10.0 + dx, 20.0))


# depth.rs:1956-1975
def test_warp_consensus_requires_similar_parallax(oracle_lib, backend):
    def agree(c, n):
        return oracle_lib.oracle_warp_decisions_agree(
            0, c[0], fptr(np.array(c[1], np.float32)), fptr(np.array(c[2], np.float32)),
            n[0], fptr(np.array(n[1], np.float32)), fptr(np.array(n[2], np.float32)))
    assert agree(_refined(2.0), _refined(4.5))
    assert not agree(_refined(2.0), _refined(6.0))
    assert not agree(_refined(2.0), (abi.NW_GLOBAL, (10.0, 20.0), (10.0, 20.0)))

    kind = np.full(9, abi.NW_GLOBAL, np.uint8)
    glob = np.tile(np.array([10.0, 20.0], np.float32), 9)
    point = glob.copy()
    measured = np.ones(9, np.uint8)
    kind[4] = abi.NW_REFINED
    point[8:10] = (12.0, 20.0)
    k, _, _ = backend.warp_filter(kind, glob, point, measured, np.zeros(9, np.float32), 3, 3,
                                  consensus=True, boundaries=False)
    assert k[4] == abi.NW_GLOBAL


# depth.rs:1978-1999
def test_warp_boundary_suppression_requires_an_image_edge(backend):
    kind = np.full(2, abi.NW_REFINED, np.uint8)
    glob = np.array([10.0, 20.0, 10.0, 20.0], np.float32)
    point = np.array([10.0, 20.0, 14.0, 20.0], np.float32)
    measured = np.ones(2, np.uint8)
    k, _, _ = backend.warp_filter(kind, glob, point, measured, np.array([1.0, 1.1], np.float32), 2, 1,
                                  consensus=False, boundaries=True)
    assert np.all(k == abi.NW_REFINED)
    k, _, _ = backend.warp_filter(kind, glob, point, measured, np.array([1.0, 1.5], np.float32), 2, 1,
                                  consensus=False, boundaries=True)
    assert np.all(k == abi.NW_BOUNDARY)


# depth.rs:2002-2014
def test_confident_global_label_is_not_treated_as_a_completion_hole(backend):
    out = backend.select_depths([NaN, 10_000.0, 2_000.0], [0.9, 0.7, 0.6], [0.4, 1.2, 1.6], [1], DepthOptions())
    assert out["has"][0] == 0
    assert out["fillable"][0] == 0


# depth.rs:2017-2029
def test_sgm_supported_ambiguous_depth_is_kept_as_regularized(backend):
    out = backend.select_depths([NaN, 100_000.0, 10_000.0, 2_000.0], [0.72, 0.70, 0.68, 0.62],
                                [0.8, 0.7, 0.75, 0.9], [1], DepthOptions())
    assert out["has"][0] == 1 and out["regularized"][0] == 1
    assert out["fillable"][0] == 0


def _kat_map():
    return DenseDepthMap(4, 1, 32, 500.0, 100_000.0,
                         depth=np.array([NaN, NaN, 500.0, 100_000.0]),
                         confidence=np.array([0.0, 1.0, 1.0, 0.0], np.float32),
                         provenance=np.array([abi.UNSUPPORTED, abi.GLOBAL, abi.MEASURED, abi.REGULARIZED],
                                             np.uint8))


def _check_diagnostics(depth, provenance, visualization):
    assert list(depth) == [0, 0, 65_535, 1]
    assert list(provenance[0:3]) == [0, 0, 0]
    assert list(provenance[3:6]) == [0, 0, 32_768]
    assert list(provenance[6:9]) == [0, 65_535, 0]
    assert provenance[9] > provenance[10]
    assert provenance[11] == 0
    assert list(visualization[0:3]) == [0, 0, 0]
    assert list(visualization[3:6]) == [0, 0, 12_000]
    assert visualization[6] > visualization[8]
    assert visualization[11] > visualization[9]


# depth.rs:2032-2075 (oracle and the host API's encoder)
def test_diagnostics_distinguish_depth_and_provenance(oracle_lib):
    m = _kat_map()
    cm = DepthMapC()
    cm.columns, cm.rows, cm.step, cm.near_depth, cm.far_depth, cm.capacity = 4, 1, 32, 500.0, 100_000.0, 4
    cm.depth, cm.confidence, cm.provenance = dptr(m.depth), fptr(m.confidence), u8ptr(m.provenance)
    depth = np.zeros(4, np.uint16)
    prov = np.zeros(12, np.uint16)
    vis = np.zeros(12, np.uint16)
    oracle_lib.oracle_diagnostic_samples(C.byref(cm), u16ptr(depth), u16ptr(prov))
    oracle_lib.oracle_visualization_samples(C.byref(cm), u16ptr(vis))
    _check_diagnostics(depth, prov, vis)
    d2, p2 = m.diagnostic_samples()
    v2 = m.visualization_samples()
    _check_diagnostics(d2, p2, v2)
    np.testing.assert_array_equal(d2, depth)
    np.testing.assert_array_equal(p2, prov)
    np.testing.assert_array_equal(v2, vis)


# depth.rs:2078-2098
def test_completion_does_not_cross_an_unsupported_region(oracle_lib):
    opt = DepthOptions(completion_iterations=8, minimum_neighbour_support=1).to_c()
    has = np.zeros(5, np.uint8)
    depth = np.zeros(5)
    conf = np.zeros(5, np.float32)
    imp = np.zeros(5, np.float32)
    reg = np.zeros(5, np.uint8)
    has[0], depth[0], conf[0], imp[0] = 1, 2_000.0, 1.0, 0.2
    guidance = np.zeros(5, np.float32)
    fillable = np.array([1, 1, 0, 1, 1], np.uint8)
    oracle_lib.oracle_complete_depth_field(u8ptr(has), dptr(depth), fptr(conf), fptr(imp), u8ptr(reg),
                                           fptr(guidance), u8ptr(fillable), 5, 1, C.byref(opt))
    assert has[1] == 1
    assert has[2] == 0 and has[3] == 0 and has[4] == 0


# depth.rs:2101-2113
def test_direct_consistency_rejects_an_island_without_filling_holes(backend):
    has = np.array([1, 0, 1], np.uint8)
    depth = np.array([2_000.0, NaN, 500.0])
    conf = np.full(3, 0.6, np.float32)
    out = backend.reject_isolated(has, depth, conf, np.full(3, 0.5, np.float32), 3, 1, 1.0e-4)
    assert np.all(out == 0)


# depth.rs:2116-2140
def test_direct_component_filter_removes_speckles_without_growing_surfaces(backend):
    has = np.zeros(36, np.uint8)
    depth = np.full(36, NaN)
    for row in range(2, 5):
        for column in range(1, 4):
            has[row * 6 + column] = 1
            depth[row * 6 + column] = 2_000.0
    for i in (3 * 6 + 5, 4 * 6 + 5):
        has[i] = 1
        depth[i] = 2_000.0
    out = backend.reject_small_components(has, depth, np.full(36, 0.5, np.float32), 6, 6, 1.0e-4, 6)
    assert out.sum() == 9
    assert out[3 * 6 + 2] == 1
    assert out[3 * 6 + 5] == 0 and out[4 * 6 + 5] == 0


# depth.rs:2143-2154
def test_direct_depth_must_improve_on_the_global_warp(oracle_lib):
    depths = np.array([10_000.0, 9_000.0, 8_000.0, 7_000.0, 6_000.0])
    scores = np.array([0.60, 0.65, 0.90, 0.65, 0.60], np.float32)
    opt = DepthOptions().to_c()
    d, c, i = C.c_double(), C.c_float(), C.c_float()
    args = (dptr(depths), fptr(scores), 5)
    assert oracle_lib.oracle_select_direct_depth(*args, 1, np.float32(0.899), 0, C.byref(opt), C.byref(d),
                                                 C.byref(c), C.byref(i)) == 0
    assert oracle_lib.oracle_select_direct_depth(*args, 1, np.float32(0.89), 0, C.byref(opt), C.byref(d),
                                                 C.byref(c), C.byref(i)) == 1


# depth.rs:2157-2171
def test_local_plane_fit_updates_only_existing_measurements(backend):
    has = np.array([0 if i == 12 else 1 for i in range(25)], np.uint8)
    depth = np.array([1.0 / (0.000_2 + (i % 5) * 0.000_001) for i in range(25)])
    depth[12] = NaN
    out = backend.fit_local_planes(has, depth, np.ones(25, np.float32), np.full(25, 0.5, np.float32), 5, 5,
                                   0.000_1)
    assert np.isnan(out[12])
    assert np.all(np.isfinite(out[has == 1]))


# align.rs:895-905 (oracle and host Warp.map)
def test_warp_grid_interpolates_and_reports_magnification(oracle_lib):
    warp = Warp.from_fn(100, 60, 10, lambda p: (np.stack([p[:, 0] * 2.0 + 1.0, p[:, 1] * 2.0 - 1.0], -1),
                                                 np.ones(len(p), bool)))
    assert (warp.columns, warp.rows) == (11, 7)
    cw = WarpC(step=10, columns=11, rows=7, points=fptr(warp.points), confidence=fptr(warp.confidence),
               capacity=77)
    q = np.zeros(2, np.float32)
    assert oracle_lib.oracle_warp_map(C.byref(cw), 25.0, 13.0, fptr(q)) == 1
    assert abs(q[0] - 51.0) < 1e-4 and abs(q[1] - 25.0) < 1e-4
    mag = C.c_float()
    assert oracle_lib.oracle_warp_magnification(C.byref(cw), 20.0, 20.0, C.byref(mag)) == 1
    assert abs(mag.value - 2.0) < 1e-4
    hq, ok = warp.map(25.0, 13.0)
    assert ok and np.array_equal(hq, q)
    partial = Warp.from_fn(100, 60, 10, lambda p: (p, p[:, 0] < 50.0))
    pw = WarpC(step=10, columns=11, rows=7, points=fptr(partial.points), confidence=fptr(partial.confidence),
               capacity=77)
    assert oracle_lib.oracle_warp_map(C.byref(pw), 10.0, 10.0, fptr(q)) == 1
    assert oracle_lib.oracle_warp_map(C.byref(pw), 90.0, 10.0, fptr(q)) == 0
    assert partial.map(10.0, 10.0)[1] and not partial.map(90.0, 10.0)[1]


def _distortion_camera():
    return ResolvedCamera(width=4160, height=3120, k=np.array([[3380.0, 0, 2080.0], [0, 3380.0, 1560.0], [0, 0, 1]]),
                          distortion=PolynomialDistortion((2080.0, 1560.0), (3380.0, 3380.0),
                                                          (0.1138, -0.3495, 0.0, 0.0, 0.0934)),
                          rotation_wc=np.eye(3), translation_wc=np.zeros(3))


# geometry.rs:367-393
def test_distortion_round_trips(oracle_lib):
    cam = _distortion_camera().to_c()
    for pixel in ([100.0, 100.0], [2080.0, 1560.0], [4100.0, 3000.0], [0.0, 3119.0]):
        ideal = np.zeros(2)
        back = np.zeros(2)
        oracle_lib.oracle_undistort(C.byref(cam), dptr(np.array(pixel)), dptr(ideal))
        oracle_lib.oracle_distort(C.byref(cam), dptr(ideal), dptr(back))
        assert abs(back[0] - pixel[0]) < 1e-6 and abs(back[1] - pixel[1]) < 1e-6


# math.rs:141-160 (host camera-model algebra)
def test_inverse_and_rotation_are_consistent():
    r = rotation_about_axis([0.3, -0.2, 0.9], 0.7)
    inv = inverse(r)
    product = r @ inv
    assert np.all(np.abs(product - IDENTITY) < 1e-12)
    assert np.all(np.abs(inv - r.T) < 1e-12)
    assert abs(determinant(r) - 1.0) < 1e-12
