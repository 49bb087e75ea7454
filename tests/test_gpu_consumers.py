"""The stage's outputs read back on the device as synthesis reads them: Warp::map,
Warp::confidence (align.rs:84-131) and DenseDepthMap::sample_nearest (depth.rs:152-159)
over batches of query points, bit for bit against the oracle, with negative, NaN,
infinite, tie-rounding and out-of-grid queries."""
import ctypes as C

import numpy as np
import pytest
import torch

from chiaro_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _queries(width, height, step, rng, n=3000):
    xy = np.stack([rng.uniform(-40, width + 40, n), rng.uniform(-40, height + 40, n)], axis=1).astype(np.float32)
    specials = [(-0.0, 0.0), (0.0, 0.0), (-1e-7, 5.0), (np.nan, 3.0), (3.0, np.nan), (np.inf, 1.0), (1.0, -np.inf),
                (step * 2.5, step * 0.5), (step * 3.5, step * 1.5), (width, height), (width + step, 0.0),
                (step * 1e6, 1.0), (step * 0.49999997, step * 2.5000002)]
    xy[:len(specials)] = np.array(specials, np.float32)
    return xy


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_warp_map_and_confidence_match_the_oracle(gpu_ctx, oracle_lib):
    rng = np.random.default_rng(5)
    sc = scenes.workload("small", seed=1)
    for t, with_confidence in ((1, True), (2, False)):
        w = sc.warps[t]
        points = np.ascontiguousarray(w.points, np.float32).copy()
        points[rng.random(len(points)) < 0.1] = np.nan  # undefined nodes
        confidence = rng.uniform(-0.2, 1.3, len(points)).astype(np.float32)
        dp, dc = _dev(points), _dev(confidence)
        dw = abi.WarpC(step=w.step, columns=w.columns, rows=w.rows,
                       points=C.cast(C.c_void_p(dp.data_ptr()), C.POINTER(C.c_float)),
                       confidence=C.cast(C.c_void_p(dc.data_ptr()) if with_confidence else None,
                                         C.POINTER(C.c_float)), capacity=w.columns * w.rows)
        xy = _queries(sc.width, sc.height, w.step, rng)
        dxy = _dev(xy)
        mapped = torch.empty((len(xy), 2), dtype=torch.float32, device="cuda")
        conf = torch.empty(len(xy), dtype=torch.float32, device="cuda")
        gpu_ctx.check(gpu_ctx.lib.chiaro_warp_sample_device(gpu_ctx.handle, C.byref(dw), dxy.data_ptr(), len(xy),
                                                            mapped.data_ptr(), conf.data_ptr()))
        mapped, conf = mapped.cpu().numpy(), conf.cpu().numpy()
        hw = abi.WarpC(step=w.step, columns=w.columns, rows=w.rows, points=points.ctypes.data_as(C.POINTER(C.c_float)),
                       confidence=confidence.ctypes.data_as(C.POINTER(C.c_float)) if with_confidence else None,
                       capacity=w.columns * w.rows)
        out = np.zeros(2, np.float32)
        for i, (x, y) in enumerate(xy):
            ok = oracle_lib.oracle_warp_map(C.byref(hw), x, y, out.ctypes.data_as(C.POINTER(C.c_float)))
            want = out if ok else np.array([np.nan, np.nan], np.float32)
            assert np.array_equal(mapped[i].view(np.uint32), want.view(np.uint32)), (i, x, y)
            c = np.float32(oracle_lib.oracle_warp_confidence(C.byref(hw), x, y))
            # bit for bit, except that a NaN's payload is the platform's (the device's canonical NaN)
            assert (np.isnan(conf[i]) and np.isnan(c)) or conf[i].view(np.uint32) == c.view(np.uint32), (i, x, y)


@pytest.mark.parametrize("step", [4, 8, 0])
def test_sample_nearest_matches_the_oracle(gpu_ctx, oracle_lib, step):
    rng = np.random.default_rng(step + 1)
    columns, rows = 61, 47
    n = columns * rows
    depth = rng.uniform(500, 20000, n)
    depth[rng.random(n) < 0.2] = np.nan
    confidence = rng.uniform(0, 1, n).astype(np.float32)
    provenance = rng.integers(0, 4, n).astype(np.uint8)
    dd, dc, dpv = _dev(depth), _dev(confidence), _dev(provenance)
    dmap = abi.DepthMapC(columns=columns, rows=rows, step=step, capacity=n,
                         depth=C.cast(C.c_void_p(dd.data_ptr()), C.POINTER(C.c_double)),
                         confidence=C.cast(C.c_void_p(dc.data_ptr()), C.POINTER(C.c_float)),
                         provenance=C.cast(C.c_void_p(dpv.data_ptr()), C.POINTER(C.c_uint8)))
    xy = _queries(columns * max(step, 1), rows * max(step, 1), max(step, 1), rng)
    dxy = _dev(xy)
    out_depth = torch.empty(len(xy), dtype=torch.float64, device="cuda")
    out_conf = torch.empty(len(xy), dtype=torch.float32, device="cuda")
    out_prov = torch.empty(len(xy), dtype=torch.uint8, device="cuda")
    out_node = torch.empty(len(xy), dtype=torch.int64, device="cuda")
    gpu_ctx.check(gpu_ctx.lib.chiaro_depth_sample_nearest_device(
        gpu_ctx.handle, C.byref(dmap), dxy.data_ptr(), len(xy), out_depth.data_ptr(), out_conf.data_ptr(),
        out_prov.data_ptr(), out_node.data_ptr()))
    node = out_node.cpu().numpy()
    hmap = abi.DepthMapC(columns=columns, rows=rows, step=step, capacity=n)
    want = np.array([oracle_lib.oracle_sample_nearest(C.byref(hmap), x, y) for x, y in xy], np.int64)
    assert np.array_equal(node, want)
    found = want >= 0
    if step == 0:
        assert not found.any()
    else:
        assert found.sum() > 1000
    assert np.array_equal(out_depth.cpu().numpy()[found].view(np.uint64), depth[want[found]].view(np.uint64))
    assert np.array_equal(out_conf.cpu().numpy()[found], confidence[want[found]])
    assert np.array_equal(out_prov.cpu().numpy()[found], provenance[want[found]])
    assert np.isnan(out_depth.cpu().numpy()[~found]).all() and (out_prov.cpu().numpy()[~found] == 0).all()
