"""The oracle's cost volume on cases whose scores follow from warped_patch_zncc's
formula (depth.rs:1772-1822) without running any restatement of it (CPU).

See ``zncc_cases``: a target that is the reference's own camera and plane scaled by
2 scores exactly 1.0 at every label, the negated plane exactly -1.0, a zero plane
None everywhere, and a node whose taps leave the plane None. The GPU stage is
checked against the same expectations in ``test_gpu_zncc_pins.py``.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200.abi import fptr, u8ptr
from chiaro_b200.depth import output_shape, pack_views

import zncc_cases


def _bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


@pytest.mark.parametrize("kind", zncc_cases.KINDS)
def test_oracle_cost_volume_on_formula_cases(kind):
    from oracle import oracle
    inputs, alignments, options = zncc_cases.self_pair(kind)
    _, (columns, rows, _) = output_shape(inputs[0].width, inputs[0].height, options)
    n, d = columns * rows, options.planes + 1
    views, keep = pack_views(inputs, alignments())
    scores = np.empty(n * d, np.float32)
    costs = np.empty(n * d, np.float32)
    guidance = np.empty(n, np.float32)
    tested = np.empty(n, np.uint8)
    opt = options.to_c()
    st = oracle.lib().oracle_build_cost_volume(views, 2, 0, C.byref(opt), 0, rows, fptr(scores), fptr(costs),
                                               fptr(guidance), u8ptr(tested), 2)
    assert st == 0
    e_scores, e_costs, e_tested = zncc_cases.expected_volume(kind, inputs, options)
    assert np.array_equal(tested, e_tested)
    assert _bits_equal(np.nan_to_num(scores, nan=9.0), np.nan_to_num(e_scores, nan=9.0))
    assert _bits_equal(costs, e_costs)
    if kind != "zero":
        assert 0.3 < e_tested.mean() < 1.0  # some nodes score, border nodes do not
