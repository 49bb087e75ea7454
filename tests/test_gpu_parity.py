"""GPU parity: the CUDA stage against the CPU oracle, bit for bit.

Every comparison is exact (bitwise for floats, equality for masks and
indices): the kernels restate the reference's arithmetic in its order, so
there is no tolerance to state. Each test runs the same seeded inputs through
the C ABI and through the oracle.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import abi, scenes
from chiaro_b200.depth import DepthOptions, output_shape, refine_multiview_depth

from backends import GpuBackend, OracleBackend

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    if a.dtype == np.float32:
        return np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if a.dtype == np.float64:
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return np.array_equal(a, b)


def assert_bits(a, b, what):
    if not bits_equal(a, b):
        a = np.asarray(a)
        b = np.asarray(b)
        if a.dtype.kind == "f":
            diff = ~((a == b) | (np.isnan(a) & np.isnan(b)))
        else:
            diff = a != b
        idx = np.flatnonzero(diff)
        raise AssertionError(f"{what}: {len(idx)} of {a.size} differ; first {idx[:5]}: "
                             f"gpu {a.ravel()[idx[:5]]} oracle {b.ravel()[idx[:5]]}")


@pytest.fixture(scope="module")
def gpu(gpu_ctx):
    return GpuBackend(gpu_ctx)


@pytest.fixture(scope="module")
def cpu():
    return OracleBackend()


@pytest.mark.parametrize("columns,rows,labels", [(1, 1, 3), (5, 1, 4), (1, 7, 33), (13, 9, 65), (40, 31, 97),
                                                 (31, 40, 129), (17, 23, 193), (9, 5, 256),
                                                 (70, 3, 40), (2, 75, 129)])
def test_sgm_bit_exact(gpu, cpu, columns, rows, labels):
    rng = np.random.default_rng(columns * 1000 + rows * 10 + labels)
    costs = rng.uniform(0, 2.25, columns * rows * labels).astype(np.float32)
    costs[rng.random(costs.size) < 0.05] = np.float32(2.25)
    guidance = rng.uniform(0, 7, columns * rows).astype(np.float32)
    assert_bits(gpu.sgm(costs, guidance, columns, rows, labels),
                cpu.sgm(costs, guidance, columns, rows, labels), "sgm")


def test_select_depths_bit_exact(gpu, cpu):
    rng = np.random.default_rng(11)
    n, D = 5000, 65
    labels = np.concatenate([[np.nan], 1.0 / np.linspace(1 / 400, 1 / 25000, D - 1)[::-1]])
    scores = rng.uniform(-0.2, 1.0, n * D).astype(np.float32)
    scores[rng.random(scores.size) < 0.1] = np.nan
    reg = rng.uniform(0, 8, n * D).astype(np.float32)
    reg[::7] = reg[::7].round(1)  # ties
    tested = (rng.random(n) < 0.9).astype(np.uint8)
    for opt in (DepthOptions(), DepthOptions(minimum_score=0.2, minimum_margin=0.05)):
        a = gpu.select_depths(labels, scores, reg, tested, opt)
        b = cpu.select_depths(labels, scores, reg, tested, opt)
        for k in ("has", "fillable", "regularized"):
            assert_bits(a[k], b[k], k)
        m = b["has"] == 1
        for k in ("depth", "confidence", "improvement"):
            assert_bits(a[k][m], b[k][m], k)


def _random_field(rng, columns, rows):
    n = columns * rows
    has = (rng.random(n) < 0.7).astype(np.uint8)
    base = 1.0 / rng.choice([800.0, 2000.0, 6000.0], size=n)
    depth = 1.0 / (base + rng.normal(0, 2e-6, n))
    conf = rng.uniform(0.3, 1.0, n).astype(np.float32)
    guidance = rng.uniform(0, 1.2, n).astype(np.float32)
    return has, depth, conf, guidance


@pytest.mark.parametrize("columns,rows", [(3, 1), (41, 31), (120, 90)])
def test_filters_bit_exact(gpu, cpu, columns, rows):
    rng = np.random.default_rng(columns)
    has, depth, conf, guidance = _random_field(rng, columns, rows)
    tol = 2.5e-6
    a = gpu.reject_isolated(has, depth, conf, guidance, columns, rows, tol)
    b = cpu.reject_isolated(has, depth, conf, guidance, columns, rows, tol)
    assert_bits(a, b, "isolated")
    a2 = gpu.reject_small_components(b, depth, guidance, columns, rows, tol, 24)
    b2 = cpu.reject_small_components(b, depth, guidance, columns, rows, tol, 24)
    assert_bits(a2, b2, "components")
    a3 = gpu.fit_local_planes(b2, depth, conf, guidance, columns, rows, 4e-6)
    b3 = cpu.fit_local_planes(b2, depth, conf, guidance, columns, rows, 4e-6)
    m = b2 == 1
    assert_bits(a3[m], b3[m], "plane fit")


def test_warp_filter_bit_exact(gpu, cpu):
    rng = np.random.default_rng(3)
    columns, rows = 60, 45
    n = columns * rows
    kind = rng.choice([abi.NW_UNDEFINED, abi.NW_GLOBAL, abi.NW_REFINED, abi.NW_OCCLUDED], size=n,
                      p=[0.05, 0.25, 0.6, 0.1]).astype(np.uint8)
    glob = rng.uniform(0, 400, 2 * n).astype(np.float32)
    point = (glob + rng.normal(0, 2.0, 2 * n)).astype(np.float32)
    measured = (rng.random(n) < 0.7).astype(np.uint8)
    guidance = rng.uniform(0, 1, n).astype(np.float32)
    a = gpu.warp_filter(kind, glob, point, measured, guidance, columns, rows)
    b = cpu.warp_filter(kind, glob, point, measured, guidance, columns, rows)
    assert_bits(a[0], b[0], "kind")


def _run_both(scene, options=None, reference_index=0, inputs=None, alignments=None):
    from oracle import oracle
    inputs = inputs if inputs is not None else scene.inputs()
    options = options or scene.options
    ref = inputs[reference_index]
    (columns, rows, step), (cc, cr, cs) = output_shape(ref.width, ref.height, options)
    n = len(inputs)
    dbg_g = oracle.debug_buffers(n, cc * cr, options.planes + 1, columns * rows)
    dbg_o = oracle.debug_buffers(n, cc * cr, options.planes + 1, columns * rows)
    al_g = alignments() if alignments else scene.alignments()
    al_o = alignments() if alignments else scene.alignments()
    dmap = refine_multiview_depth(inputs, reference_index, al_g, options, debug=dbg_g)
    omap = oracle.refine_multiview_depth(inputs, reference_index, al_o, options, threads=8, debug=dbg_o)
    return dmap, omap, al_g, dbg_g, dbg_o


STAGES = ["coarse_tested", "coarse_guidance", "coarse_scores", "coarse_costs", "regularised", "coarse_has",
          "coarse_fillable", "coarse_regularized", "direct_tested", "direct_guidance", "direct_has",
          "isolated_has", "component_has"]


def _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, n_views):
    for k in STAGES:
        assert_bits(dbg_g[k], dbg_o[k], k)
    m = dbg_o["coarse_has"] == 1
    for k in ("coarse_depth", "coarse_confidence", "coarse_improvement"):
        assert_bits(dbg_g[k][m], dbg_o[k][m], k)
    m = dbg_o["direct_has"] == 1
    for k in ("direct_depth", "direct_confidence", "direct_improvement"):
        assert_bits(dbg_g[k][m], dbg_o[k][m], k)
    m = dbg_o["component_has"] == 1
    assert_bits(dbg_g["fitted_depth"][m], dbg_o["fitted_depth"][m], "fitted_depth")
    assert_bits(dbg_g["decision_kind"], dbg_o["decision_kind"], "decision kinds")
    assert_bits(dmap.depth, omap["depth"], "map depth")
    assert_bits(dmap.confidence, omap["confidence"], "map confidence")
    assert_bits(dmap.provenance, omap["provenance"], "map provenance")
    for t in range(n_views):
        rep = omap["reports"][t]
        if not rep.present:
            assert al_g[t].report.depth is None
            continue
        assert al_g[t].report.depth is not None
        assert_bits(al_g[t].warp.points.reshape(-1), omap["points"][t], f"warp points {t}")
        assert_bits(al_g[t].warp.confidence, omap["warp_confidence"][t], f"warp confidence {t}")
        r = al_g[t].report.depth
        for f in ("tested_nodes", "measured_nodes", "regularized_nodes", "fallback_nodes", "refined_nodes",
                  "occluded_nodes", "boundary_nodes"):
            assert getattr(r, f) == getattr(rep, f), f
        assert np.float32(r.refined_fraction) == np.float32(rep.refined_fraction)
        assert (r.median_depth is None) == (not rep.has_median_depth)
        if r.median_depth is not None:
            assert r.median_depth == rep.median_depth
            assert np.float32(r.median_score_improvement) == np.float32(rep.median_score_improvement)


@pytest.mark.parametrize("name,seed", [("tiny", 1), ("tiny", 2), ("small", 1), ("small", 3)])
def test_stage_bit_exact(name, seed):
    sc = scenes.workload(name, seed=seed)
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc)
    assert dmap is not None and omap is not None
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))
    assert (dmap.provenance == abi.MEASURED).sum() > 0.3 * dmap.provenance.size


def test_stage_two_view_options_bit_exact():
    sc = scenes.workload("tiny", seed=5, n_sources=1, horizontal_only=True,
                         options=dict(minimum_support=1, best_view_count=1, planes=20))
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


def test_stage_with_completion_and_grid_step_bit_exact():
    sc = scenes.workload("tiny", seed=6)
    opt = DepthOptions(**{**sc.options.__dict__, "completion_iterations": 3, "minimum_neighbour_support": 1,
                          "grid_step": 12, "patch_radius": 3})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


@pytest.mark.parametrize("grid_step", [5, 10])
def test_stage_with_an_odd_grid_step_bit_exact(grid_step):
    """An odd step puts taps off the even tap lattice: grid_step 5 gives an odd coarse step
    (the cost volume samples the planes per tap) and an even fine step (the direct pass and
    the decisions read the lattice); grid_step 10 the other way round."""
    sc = scenes.workload("tiny", seed=7)
    opt = DepthOptions(**{**sc.options.__dict__, "grid_step": grid_step})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


def test_stage_two_view_full_size_bit_exact():
    """The two-view workload at its full size (1040x780, one source at 25 mm, 64 planes,
    minimum_support = best_view_count = 1): the whole stage against the oracle."""
    sc = scenes.workload("two_view", seed=0)
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))
    assert (dmap.provenance == abi.MEASURED).sum() > 0.3 * dmap.provenance.size


def test_stage_with_seven_targets_bit_exact():
    """Seven sources: each decision phase lists 42 and 56 items (two rounds of a warp), a
    direct-pass node up to 98, and the tap lattice holds eight planes."""
    sc = scenes.workload("tiny", seed=9, n_sources=7)
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


def test_stage_with_a_wide_patch_bit_exact():
    """patch_radius 6: the wide retry's radius is 12 (25 x 25 taps), so border nodes read the
    tap lattice out to its full margin."""
    sc = scenes.workload("tiny", seed=8)
    opt = DepthOptions(**{**sc.options.__dict__, "patch_radius": 6})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


@pytest.mark.parametrize("radius", [1, 2])
def test_stage_with_a_narrow_patch_bit_exact(radius):
    """patch_radius 1 and 2: the direct pass works at radius 3 and reads the reference patches
    computed at that radius, while the decisions, at the smaller radius, sum their own."""
    sc = scenes.workload("tiny", seed=10 + radius)
    opt = DepthOptions(**{**sc.options.__dict__, "patch_radius": radius})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


@pytest.mark.parametrize("sources,radius", [(2, 2), (3, 3)])
def test_stage_with_two_and_three_targets_bit_exact(sources, radius):
    """Two targets take the CTA-pooled decisions (12 and 16 items per node), three the
    per-warp form (18 and 24 items); with the narrow radius the decisions sum their own
    patches, with radius 3 they read the precomputed ones."""
    sc = scenes.workload("tiny", seed=20 + sources, n_sources=sources)
    opt = DepthOptions(**{**sc.options.__dict__, "patch_radius": radius})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))


def test_stage_at_the_finest_coarse_grid_bit_exact():
    """grid_step 4: the coarse grid at the direct grid's step (the finest the reference
    reaches, depth.rs:326-328), as in the five-view workload's step-4 configuration."""
    sc = scenes.workload("small", seed=4)
    opt = DepthOptions(**{**sc.options.__dict__, "grid_step": 4})
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, options=opt)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))
    assert (dmap.provenance == abi.MEASURED).sum() > 0.3 * dmap.provenance.size


def test_stage_with_unaccepted_uncalibrated_and_partial_warps():
    sc = scenes.workload("tiny", seed=7, n_sources=3)
    inputs = sc.inputs()
    inputs[2].camera = None  # a module without calibration is skipped (depth.rs:1575-1579)

    def alignments():
        al = sc.alignments()
        al[3].report.accepted = False  # rejected module: untouched (depth.rs:420-426)
        pts = al[1].warp.points.reshape(al[1].warp.rows, al[1].warp.columns, 2)
        pts[:, -2:] = np.nan  # undefined mapping near the right edge
        return al

    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc, inputs=inputs, alignments=alignments)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(inputs))
    assert al_g[2].report.depth is None and al_g[3].report.depth is None
    assert al_g[1].report.depth is not None


def test_none_paths_match_the_reference():
    sc = scenes.workload("tiny", seed=1)
    inputs = sc.inputs()
    assert refine_multiview_depth(inputs, 0, sc.alignments(), DepthOptions(planes=2)) is None
    assert refine_multiview_depth(inputs, 5, sc.alignments(), sc.options) is None
    assert refine_multiview_depth(inputs, 0, sc.alignments()[:2], sc.options) is None
    inputs[0].camera = None
    assert refine_multiview_depth(inputs, 0, sc.alignments(), sc.options) is None


def test_no_targets_gives_unsupported_map():
    sc = scenes.workload("tiny", seed=1)
    al = sc.alignments()
    for a in al[1:]:
        a.report.accepted = False
    dmap = refine_multiview_depth(sc.inputs(), 0, al, sc.options)
    assert dmap is not None
    assert np.all(dmap.provenance == abi.UNSUPPORTED)
    assert all(a.report.depth is None for a in al)


@pytest.mark.parametrize("name,seed,mirrors,orientation", [
    ("small", 5, {1: True, 2: False}, None),                              # both flip kinds as targets
    ("tiny", 11, {0: True}, {1: (0.03, -0.02, 0.04)}),                    # mirrored reference
    ("small", 6, {2: False}, {2: (-0.02, 0.05, 0.01), 1: (0.01, 0.01, -0.03)}),  # mirror + orientation
    ("tiny", 12, {0: False, 1: True, 2: False}, {0: (0.02, 0.0, -0.01)}),  # every module mirrored
], ids=["targets-both-flips", "mirrored-reference", "orientation-corrections", "all-mirrored"])
def test_stage_with_mirrored_modules_bit_exact(name, seed, mirrors, orientation):
    """Modules behind fold mirrors (Pose::Mirror with flip_img_around_x Some(true) and
    Some(false), geometry.rs:86-104, 129-136) and orientation corrections
    (geometry.rs:111-114): the camera branches of the L16's mid and tele modules."""
    sc = scenes.workload(name, seed=seed, mirrors=mirrors, orientation=orientation)
    assert any(c.pose_kind == 1 for c in sc.cameras)
    dmap, omap, al_g, dbg_g, dbg_o = _run_both(sc)
    _compare_stage_outputs(dmap, omap, al_g, dbg_g, dbg_o, len(sc.cameras))
    assert (dmap.provenance == abi.MEASURED).sum() > 0.2 * dmap.provenance.size
