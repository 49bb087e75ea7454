"""The GPU stage's cost volume on the formula cases of ``zncc_cases`` (GPU).

Exactly 1.0 for a target that is the reference scaled by 2, -1.0 for its negation,
None for a zero plane and for nodes whose taps leave the plane, with the costs
that follow (depth.rs:1229-1240): expectations derived from warped_patch_zncc
(depth.rs:1772-1822) alone, independent of the oracle.
"""
import numpy as np
import pytest

from chiaro_b200.depth import output_shape, refine_multiview_depth

import zncc_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", zncc_cases.KINDS)
def test_stage_cost_volume_on_formula_cases(gpu_ctx, kind):
    from oracle import oracle
    inputs, alignments, options = zncc_cases.self_pair(kind)
    ref = inputs[0]
    (columns, rows, _), (cc, cr, _) = output_shape(ref.width, ref.height, options)
    dbg = oracle.debug_buffers(2, cc * cr, options.planes + 1, columns * rows)
    dmap = refine_multiview_depth(inputs, 0, alignments(), options, context=gpu_ctx, debug=dbg)
    assert dmap is not None
    e_scores, e_costs, e_tested = zncc_cases.expected_volume(kind, inputs, options)
    assert np.array_equal(dbg["coarse_tested"], e_tested)
    got = np.nan_to_num(dbg["coarse_scores"], nan=9.0)
    assert np.array_equal(got.view(np.uint32), np.nan_to_num(e_scores, nan=9.0).view(np.uint32))
    assert np.array_equal(dbg["coarse_costs"].view(np.uint32), e_costs.view(np.uint32))
