"""Cost-volume cases whose answer follows from warped_patch_zncc's formula alone
(crates/chiaro-fusion/src/depth.rs:1772-1822), shared by the oracle test (CPU) and
the stage test (GPU).

The target module is the reference module itself: the same camera and an identity
global warp, so map_at_depth (depth.rs:1738-1759) returns the reference pixel at
every depth (up to ~1e-9 px, far below half an f32 ulp of the halved sample
coordinates), and every tap of the target reads the reference plane's position.
Its plane is the reference's plane transformed:

* ``double``  — 2 x plane. Scaling by 2 commutes with every rounding of Plane::sample
  and of the weighted sums, so covariance = E, target energy = 4 E and the
  denominator sqrt(E * 4E) = 2E: the score is exactly 1.0 (sqrt(x * x) == |x| in
  binary floating point).
* ``negated`` — -plane: covariance = -E, energy E, score exactly -1.0.
* ``zero``    — both planes 0: every energy is 0, the denominator is not above 1e-6,
  and the score is None at every node.

A node scores only when every tap's sample lies in [0, w-1] x [0, h-1] of the plane
(Plane::sample, image.rs:451-466): ``inside_mask`` states which, from the tap
arithmetic of depth.rs:1791-1795 ((p - 0.5) * 0.5 with p = centre + 2 d). Scored
nodes are tested, and their costs are clamp(1 - s, 0, 2) + 0.10 (l - 1) / (D - 2)
(depth.rs:1229-1240); the others hold NaN and MISSING_COST = 2.25.
"""
from __future__ import annotations

import numpy as np

from chiaro_b200 import scenes
from chiaro_b200.align import AlignInput, AlignmentReport, ModuleAlignment, Warp
from chiaro_b200.depth import DepthOptions, output_shape
from chiaro_b200.image import Plane

MISSING_COST = np.float32(2.25)
KINDS = ("double", "negated", "zero")


def self_pair(kind: str, seed: int = 1):
    """(inputs, alignments, options) of a reference and its transformed copy."""
    sc = scenes.workload("tiny", seed=seed)
    ref = sc.inputs()[0]
    data = ref.luminance.data.astype(np.float32)
    if kind == "double":
        target_data = data * np.float32(2.0)
    elif kind == "negated":
        target_data = -data
    else:
        data = np.zeros_like(data)
        target_data = np.zeros_like(data)
    ref_plane = Plane(ref.luminance.width, ref.luminance.height, data)
    tgt_plane = Plane(ref.luminance.width, ref.luminance.height, target_data)
    inputs = [AlignInput(name="R", luminance=ref_plane, width=ref.width, height=ref.height, camera=ref.camera,
                         nominal_focal_px=ref.nominal_focal_px),
              AlignInput(name="T", luminance=tgt_plane, width=ref.width, height=ref.height, camera=ref.camera,
                         nominal_focal_px=ref.nominal_focal_px)]

    def alignments():
        return [ModuleAlignment(name=n, warp=Warp.identity(ref.width, ref.height, 32),
                                report=AlignmentReport(camera=n, accepted=True)) for n in ("R", "T")]

    options = DepthOptions(**{**sc.options.__dict__, "minimum_support": 1, "best_view_count": 1})
    return inputs, alignments, options


def inside_mask(inputs, options) -> np.ndarray:
    """Coarse nodes whose every tap samples inside the reference plane."""
    ref = inputs[0]
    _, (columns, rows, step) = output_shape(ref.width, ref.height, options)
    r = options.patch_radius
    lw, lh = ref.luminance.width, ref.luminance.height
    xs = np.arange(columns, dtype=np.float64) * step
    ys = np.arange(rows, dtype=np.float64) * step
    lo_x = np.float32((xs - 2 * r - 0.5) * 0.5)
    hi_x = np.float32((xs + 2 * r - 0.5) * 0.5)
    lo_y = np.float32((ys - 2 * r - 0.5) * 0.5)
    hi_y = np.float32((ys + 2 * r - 0.5) * 0.5)
    ok_x = (lo_x >= 0) & (hi_x <= np.float32(lw - 1))
    ok_y = (lo_y >= 0) & (hi_y <= np.float32(lh - 1))
    return (ok_y[:, None] & ok_x[None, :]).reshape(-1)


def expected_volume(kind: str, inputs, options):
    """(scores, costs, tested) of the case, from the formula alone."""
    inside = inside_mask(inputs, options) if kind != "zero" else np.zeros(0, bool)
    ref = inputs[0]
    _, (columns, rows, _) = output_shape(ref.width, ref.height, options)
    n, d = columns * rows, options.planes + 1
    if kind == "zero":
        inside = np.zeros(n, bool)
    value = {"double": np.float32(1.0), "negated": np.float32(-1.0), "zero": np.float32(np.nan)}[kind]
    scores = np.full((n, d), np.nan, np.float32)
    scores[inside] = value
    prior = np.array([0.0] + [np.float32(0.10) * np.float32(l - 1) / np.float32(d - 2) for l in range(1, d)],
                     np.float32)
    base = np.clip(np.float32(1.0) - value, np.float32(0.0), np.float32(2.0)) if np.isfinite(value) else 0
    costs = np.full((n, d), MISSING_COST, np.float32)
    costs[inside] = (np.float32(base) + prior).astype(np.float32)
    return scores.reshape(-1), costs.reshape(-1), inside.astype(np.uint8)
