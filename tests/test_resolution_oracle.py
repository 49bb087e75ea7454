"""The oracle's refine_resolution_warp and match_patch against the reference's own
tests (resolution.rs:532-562, image.rs:658-668), and the exp restatement over the
Gaussian footprint's arguments."""
import ctypes as C

import numpy as np

from resolution_cases import F, identity_warp, kat_planes, oracle_refine, textured, warp_map


def _match(lib, reference, target, rx, ry, size, radius):
    shift = np.zeros(2, np.float32)
    score = C.c_float()
    ok = lib.oracle_match_patch(reference.ctypes.data_as(F), reference.shape[1], reference.shape[0],
                                target.ctypes.data_as(F), target.shape[1], target.shape[0], rx, ry, size, radius,
                                shift.ctypes.data_as(F), C.byref(score))
    return (shift, score.value) if ok else None


def test_patch_match_recovers_a_known_shift_with_subpixel_precision(oracle_lib):
    reference = textured(200, 160, (0.0, 0.0))
    target = textured(200, 160, (3.4, -2.6))
    found = _match(oracle_lib, reference, target, 60, 50, 48, 8)
    assert found is not None
    shift, score = found
    assert abs(shift[0] - 3.4) < 0.25 and abs(shift[1] + 2.6) < 0.25 and score > 0.9
    flat = np.zeros((160, 200), np.float32)
    assert _match(oracle_lib, flat, target, 60, 50, 48, 8) is None


def test_local_resolution_warp_recovers_a_subpixel_plane_shift(oracle_lib):
    reference, target = kat_planes((0.6, -0.35))
    width, height = 512, 384
    base = identity_warp(width, height)
    refined = oracle_refine(oracle_lib, reference, target, base, width, height)
    q = warp_map(refined.warp, 256.0, 192.0)
    assert q is not None
    assert abs(q[0] - 256.0 - 0.6 * 2.0) < 0.35 and abs(q[1] - 192.0 + 0.35 * 2.0) < 0.35
    # Warp::confidence at the node (256, 192) is that node's confidence
    assert refined.warp.confidence[(192 // 32) * refined.warp.columns + 256 // 32] > 0.5
    assert refined.report.verified_fraction > 0.5
    assert refined.report.supported_fraction >= refined.report.verified_fraction


def test_expf_matches_libm_over_the_gaussian_footprint():
    """sample_at_reference_bandwidth's exp arguments reach -13.2 (sigma 0.55, radius 2);
    the range weights' sweep covers |x| <= 8.3, this one the rest, every float."""
    from chiaro_b200 import build, runtime
    build.build()
    hc = runtime.load_hostcheck()
    bits = lambda v: int(np.array([v], np.float32).view(np.uint32)[0])
    bad = C.c_uint32(0)
    assert hc.chiaro_hc_expf_mismatches(bits(8.0), bits(13.3) + 1, 1, C.byref(bad)) == 0, hex(bad.value)
