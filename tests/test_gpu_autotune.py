"""Launch-shape autotuning of the cost volume (GPU).

Every CTA size of the cost volume lists, scores and aggregates the same items, so
each forced size must give the whole stage the oracle's bits; the autotuner keeps one
choice per (targets, labels scored, radius) bucket of at least 4096 nodes.
"""
import numpy as np
import pytest

from chiaro_b200 import scenes
from chiaro_b200.depth import DepthOptions, output_shape, refine_multiview_depth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    from oracle import oracle
    sc = scenes.workload("small", seed=8)
    opt = DepthOptions(**{**sc.options.__dict__, "grid_step": 4})  # 81 x 61 coarse nodes: tuned
    (columns, rows, _), (cc, cr, _) = output_shape(sc.width, sc.height, opt)
    dbg = oracle.debug_buffers(len(sc.cameras), cc * cr, opt.planes + 1, columns * rows)
    omap = oracle.refine_multiview_depth(sc.inputs(), 0, sc.alignments(), opt, threads=8, debug=dbg)
    return sc, opt, dbg, omap, cc * cr


@pytest.mark.parametrize("mode", [64, 96, 128, 160, 192, 1])
def test_every_cost_shape_gives_the_oracle_bits(case, mode):
    from oracle import oracle
    from chiaro_b200.runtime import DepthContext
    sc, opt, dbg_o, omap, n = case
    ctx = DepthContext(0)
    try:
        ctx.set_autotune(mode)
        (columns, rows, _), _ = output_shape(sc.width, sc.height, opt)
        dbg = oracle.debug_buffers(len(sc.cameras), n, opt.planes + 1, columns * rows)
        dmap = refine_multiview_depth(sc.inputs(), 0, sc.alignments(), opt, context=ctx, debug=dbg)
        for k in ("coarse_scores", "coarse_costs", "coarse_tested", "regularised"):
            assert np.array_equal(dbg[k].view(np.uint8), dbg_o[k].view(np.uint8)), k
        assert np.array_equal(dmap.depth.view(np.uint64), omap["depth"].view(np.uint64))
        tuning = ctx.tuning()
        if mode == 1:
            assert len(tuning) == 1 and list(tuning.values())[0] in (64, 96, 128, 160, 192)
            (targets, labels, radius), _ = next(iter(tuning.items()))
            assert (targets, labels, radius) == (2, opt.planes + 1, opt.patch_radius)
        else:
            assert tuning == {}
    finally:
        ctx.close()


def test_bad_modes_are_refused(gpu_ctx):
    from chiaro_b200 import abi
    for mode in (2, 63, 256, -1):
        assert gpu_ctx.lib.chiaro_depth_set_autotune(gpu_ctx.handle, mode) == abi.ERR_ARGUMENT
    gpu_ctx.set_autotune(1)
