"""The device math restatements against the platform libm and the oracle (CPU).

The kernels compute exp(-1.2 |dr|) range weights, the plane-fit exp and the
bilinear and camera arithmetic with code shared with a host build
(libchiaro_hostcheck.so). Bit equality with libm is what lets the GPU stage
match the reference bit for bit: these tests check it over every float in the
ranges the stage uses (in slices sized for the CPU suite; the full sweeps run
with CHIARO_EXHAUSTIVE=1).
"""
import ctypes as C
import os

import numpy as np
import pytest

from chiaro_b200 import runtime, scenes
from chiaro_b200.abi import dptr, fptr

EXHAUSTIVE = os.environ.get("CHIARO_EXHAUSTIVE") == "1"


@pytest.fixture(scope="module")
def hc():
    from chiaro_b200 import build
    build.build()
    return runtime.load_hostcheck()


def _float_bits(x: float) -> int:
    return int(np.array([x], np.float32).view(np.uint32)[0])


def test_expf_matches_libm_on_range_weights(hc):
    # range weights use x = -1.2 |dr| with |dr| <= ln(1001) ~ 6.91: x in [-8.3, 0]
    bad = C.c_uint32(0)
    hi = _float_bits(8.3)
    if EXHAUSTIVE:
        assert hc.chiaro_hc_expf_mismatches(0, hi, 1, C.byref(bad)) == 0, hex(bad.value)
    else:
        # a contiguous slice of 65536 floats at the start of every binade
        for e in range(0, hi, 0x00800000):
            assert hc.chiaro_hc_expf_mismatches(e, min(hi, e + 65536), 1, C.byref(bad)) == 0, hex(bad.value)


def test_expf_special_values(hc):
    for x in [0.0, -0.0, -103.9, -104.0, -150.0, 88.0, 89.0, float("inf"), float("-inf")]:
        a = np.float32(np.exp(np.float32(x))) if np.isfinite(x) else (np.float32(np.inf) if x > 0 else np.float32(0))
        got = np.float32(hc.chiaro_hc_exp_f32(x))
        ref = C.CDLL("libm.so.6").expf
        ref.restype = C.c_float
        ref.argtypes = [C.c_float]
        assert np.float32(ref(x)).view(np.uint32) == got.view(np.uint32), x
        del a
    assert np.isnan(hc.chiaro_hc_exp_f32(float("nan")))


def test_exp_f64_matches_libm_on_plane_fit_weights(hc):
    # plane-fit weights use exp(-2.5 * e) for every f32 e in [0, 0.6]
    bad = C.c_uint32(0)
    hi = _float_bits(0.6) + 1
    if EXHAUSTIVE:
        assert hc.chiaro_hc_exp_mismatches(0, hi, -2.5, C.byref(bad)) == 0, hex(bad.value)
    else:
        for e in range(0, hi, 0x00800000):
            assert hc.chiaro_hc_exp_mismatches(e, min(hi, e + 8192), -2.5, C.byref(bad)) == 0, hex(bad.value)


def test_exp_f64_plane_fit_spatial_values_and_specials(hc):
    libm = C.CDLL("libm.so.6")
    libm.exp.restype = C.c_double
    libm.exp.argtypes = [C.c_double]
    # the restatement covers |x| <= 700 (the stage uses [-1.5, 0])
    for x in [0.0, -0.0, -1e-300, -0.5, -1.5, -3.0, -699.9, 1.0, 699.0]:
        assert np.float64(libm.exp(x)).view(np.uint64) == np.float64(hc.chiaro_hc_exp_f64(x)).view(np.uint64), x


def test_magic_floor_is_exact_below_2_pow_22(hc):
    # every float in [0, 2^22): the fast bilinear fetch relies on it
    hi = _float_bits(4194304.0)
    if EXHAUSTIVE:
        assert hc.chiaro_hc_floor_mismatches(0, hi) == 0
    else:
        for e in range(0, hi, 0x00400000):
            assert hc.chiaro_hc_floor_mismatches(e, min(hi, e + 262144)) == 0


def test_small_division_is_exact(hc):
    # the kernels' item, tap and label indices (below 2^16) are split by SmallDiv's
    # multiply instead of an integer division
    assert hc.chiaro_hc_smalldiv_mismatches() == 0


def test_register_aggregate_matches_the_sorted_form(hc):
    # the cost kernel aggregates up to 8 views with a sorting network in registers
    assert hc.chiaro_hc_aggregate_mismatches(200000, 7) == 0


def test_plane_sample_matches_oracle(hc, oracle_lib):
    rng = np.random.default_rng(3)
    data = rng.uniform(0, 7, (37, 53)).astype(np.float32)
    pts = np.concatenate([rng.uniform(-1, 54, (4000, 2)), [[0, 0], [52, 36], [52.0, 0], [-0.0, 3], [52.000004, 1]]])
    for x, y in pts.astype(np.float32):
        ok1, ok2 = C.c_int(), C.c_int()
        a = oracle_lib.oracle_plane_sample(fptr(data), 53, 37, float(x), float(y), C.byref(ok1))
        b = hc.chiaro_hc_plane_sample(fptr(data), 53, 37, float(x), float(y), C.byref(ok2))
        assert ok1.value == ok2.value
        if ok1.value:
            assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


def test_warp_map_matches_oracle(hc, oracle_lib):
    from chiaro_b200.abi import WarpC
    sc = scenes.workload("tiny", seed=2)
    w = sc.warps[1]
    pts = np.ascontiguousarray(w.points.reshape(-1))
    cw = WarpC(step=w.step, columns=w.columns, rows=w.rows, points=fptr(pts), confidence=fptr(w.confidence),
               capacity=w.columns * w.rows)
    rng = np.random.default_rng(5)
    for x, y in rng.uniform(-5, 200, (3000, 2)).astype(np.float32):
        o1 = np.zeros(2, np.float32)
        o2 = np.zeros(2, np.float32)
        a = oracle_lib.oracle_warp_map(C.byref(cw), float(x), float(y), fptr(o1))
        b = hc.chiaro_hc_warp_map(fptr(pts), w.step, w.columns, w.rows, float(x), float(y), fptr(o2))
        assert a == b
        if a:
            assert np.array_equal(o1.view(np.uint32), o2.view(np.uint32))
        q, ok = w.map(x, y)
        assert bool(ok) == bool(a)
        if a:
            assert np.array_equal(np.asarray(q, np.float32).view(np.uint32), o1.view(np.uint32))


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_camera_model_matches_oracle(hc, oracle_lib, name):
    sc = scenes.workload(name, seed=4)
    ref, tgt = sc.cameras[0].to_c(), sc.cameras[1].to_c()
    rng = np.random.default_rng(6)
    for px, py, depth in zip(rng.uniform(-50, sc.width + 50, 400), rng.uniform(-50, sc.height + 50, 400),
                             1.0 / rng.uniform(1 / 1e8, 1 / 300.0, 400)):
        pixel = np.array([px, py])
        o1, o2 = np.zeros(2), np.zeros(2)
        a = oracle_lib.oracle_map_from(C.byref(tgt), C.byref(ref), dptr(pixel), depth, dptr(o1))
        b = hc.chiaro_hc_map_from(C.byref(tgt), C.byref(ref), dptr(pixel), depth, dptr(o2))
        assert a == b
        if a:
            assert np.array_equal(o1.view(np.uint64), o2.view(np.uint64))
            # host numpy model (used for warps and rendering) agrees too
            q, ok = sc.cameras[1].map_from(sc.cameras[0], pixel[None], depth)
            assert ok[0] and np.array_equal(q[0].view(np.uint64), o1.view(np.uint64))
