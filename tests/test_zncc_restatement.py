"""An independent scalar restatement of score_one_view against the oracle (CPU).

The oracle (C++) and the kernels restate warped_patch_zncc with the same
structure, so a slip shared by both would pass every GPU parity test. This file
restates score_one_view, map_at_depth and warped_patch_zncc once more, as plain
Python loops over numpy float32 scalars (crates/chiaro-fusion/src/depth.rs:
1593-1627, 1738-1759, 1772-1822), taking Plane::sample and Warp::map from the
host API (image.rs:451-466, align.rs:84-111), the camera model from
chiaro_b200.camera, and expf from the platform libm (what Rust's f32::exp calls on
Linux). Every score must equal the oracle's bit for bit, over seeded centres and
label depths of a rendered scene with distortion, mirror modules and an
orientation correction, at two patch radii.
"""
import ctypes as C
import ctypes.util

import numpy as np
import pytest

from chiaro_b200 import scenes
from chiaro_b200.depth import pack_views

F = np.float32
INFINITY_DEPTH = 1.0e8  # depth.rs:23

_libm = C.CDLL(ctypes.util.find_library("m"))
_libm.expf.restype = C.c_float
_libm.expf.argtypes = [C.c_float]


def expf(x):
    return F(_libm.expf(float(x)))


def fmax0(v):
    """f32::max(v, 0.0): NaN gives 0."""
    return F(0.0) if not (v >= F(0.0)) else v


def warp_map(warp, x, y):
    q, ok = warp.map(np.array([x], np.float32), np.array([y], np.float32))
    return (q[0, 0], q[0, 1]) if ok[0] else None


def map_at_depth(ref_cam, tgt_cam, warp, pixel, depth):
    gq = warp_map(warp, F(pixel[0]), F(pixel[1]))
    if gq is None:
        return None
    corrected, ok = ref_cam.map_from(tgt_cam, np.array([[float(gq[0]), float(gq[1])]]), INFINITY_DEPTH)
    if not ok[0]:
        return None
    q, ok = tgt_cam.map_from(ref_cam, corrected, depth)
    if not ok[0] or not np.isfinite(q[0]).all():
        return None
    return float(q[0, 0]), float(q[0, 1])


def warped_patch_zncc(ref_plane, tgt_plane, warp, centre, delta, radius):
    centre_reference = ref_plane.sample(F((centre[0] - 0.5) * 0.5), F((centre[1] - 0.5) * 0.5))
    if centre_reference is None:
        return None
    sigma = max(F(radius) * F(0.75), F(1.0))
    count = sum_r = sum_t = sum_rr = sum_tt = sum_rt = F(0.0)
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            p = (centre[0] + dx * 2.0, centre[1] + dy * 2.0)
            rv = ref_plane.sample(F((p[0] - 0.5) * 0.5), F((p[1] - 0.5) * 0.5))
            if rv is None:
                return None
            gq = warp_map(warp, F(p[0]), F(p[1]))
            if gq is None:
                return None
            q = (float(gq[0]) + delta[0], float(gq[1]) + delta[1])
            tv = tgt_plane.sample(F((q[0] - 0.5) * 0.5), F((q[1] - 0.5) * 0.5))
            if tv is None:
                return None
            distance_sq = F(dx * dx + dy * dy)
            spatial = expf(-distance_sq / (F(2.0) * sigma * sigma))
            range_weight = expf(F(-1.2) * abs(rv - centre_reference))
            w = spatial * range_weight
            count = count + w
            sum_r = sum_r + w * rv
            sum_t = sum_t + w * tv
            sum_rr = sum_rr + w * rv * rv
            sum_tt = sum_tt + w * tv * tv
            sum_rt = sum_rt + w * rv * tv
    covariance = sum_rt - sum_r * sum_t / count
    reference_energy = sum_rr - sum_r * sum_r / count
    target_energy = sum_tt - sum_t * sum_t / count
    denominator = np.sqrt(fmax0(reference_energy) * fmax0(target_energy))
    if not denominator > F(1.0e-6):
        return None
    return min(max(covariance / denominator, F(-1.0)), F(1.0))


def score_one_view(ref, tgt, warp, centre, depth, radius):
    gc = warp_map(warp, F(centre[0]), F(centre[1]))
    if gc is None:
        return None
    if depth is None:
        mapped = (float(gc[0]), float(gc[1]))
    else:
        mapped = map_at_depth(ref.camera, tgt.camera, warp, centre, depth)
        if mapped is None:
            return None
    delta = (mapped[0] - float(gc[0]), mapped[1] - float(gc[1]))
    if abs(delta[0]) > 128.0 or abs(delta[1]) > 128.0:
        return None
    return warped_patch_zncc(ref.luminance, tgt.luminance, warp, centre, delta, radius)


@pytest.fixture(scope="module")
def scene():
    return scenes.workload("small", seed=2, mirrors={2: True}, orientation={1: (0.02, -0.01, 0.03)})


@pytest.mark.parametrize("radius", [2, 4])
def test_scalar_restatement_equals_the_oracle(scene, radius):
    from oracle import oracle
    inputs, alignments = scene.inputs(), scene.alignments()
    views, keep = pack_views(inputs, alignments)
    rng = np.random.default_rng(radius)
    depths = [None] + list(1.0 / np.linspace(1 / 400.0, 1 / 20000.0, 24))
    scored = nones = 0
    for _ in range(70):
        centre = (float(rng.integers(0, 41) * 8), float(rng.integers(0, 31) * 8))
        depth = depths[int(rng.integers(0, len(depths)))]
        t = int(rng.integers(1, len(inputs)))
        expected = score_one_view(inputs[0], inputs[t], alignments[t].warp, centre, depth, radius)
        out = C.c_float()
        ok = oracle.lib().oracle_score_one_view(views, len(inputs), 0, t, centre[0], centre[1],
                                                np.nan if depth is None else depth, radius, C.byref(out))
        assert ok == (expected is not None), (centre, depth, t)
        if ok:
            assert np.float32(out.value).view(np.uint32) == np.float32(expected).view(np.uint32), \
                (centre, depth, t, out.value, expected)
            scored += 1
        else:
            nones += 1
    assert scored > 30 and nones > 0
