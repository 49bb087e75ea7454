"""Golden fixtures of the whole depth stage: self-contained inputs and outputs.

Each ``<name>.npz`` holds a seeded scene's inputs in the C ABI's own form
(luminance planes, warp grids, the ``chiaro_camera`` and ``chiaro_depth_options``
structs as raw bytes) and the oracle's outputs for them (depth map, per-target
refined warps and report counters, the coarse and fine fields, the decision
kinds). ``make_golden.py`` writes them; the CPU tests pin the oracle to them and
the GPU tests check the CUDA stage against them directly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from chiaro_b200 import abi
from chiaro_b200.abi import CameraC, DepthMapC, DepthOptionsC, DepthReportC, ViewC, WarpC, dptr, fptr, u8ptr

HERE = Path(__file__).resolve().parent
NAMES = ["tiny_seed2", "small_seed5"]
REPORT_FIELDS = ["present", "has_median_depth", "tested_nodes", "measured_nodes", "regularized_nodes",
                 "fallback_nodes", "refined_nodes", "occluded_nodes", "boundary_nodes", "reconstructed_fraction",
                 "refined_fraction", "occluded_fraction", "has_median_score_improvement"]
DEBUG_FIELDS = ["coarse_has", "coarse_depth", "direct_has", "component_has", "decision_kind"]


def load(name: str) -> dict:
    with np.load(HERE / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def views_of(g: dict):
    """The chiaro_view array of a fixture (keep the second value alive while the views are used)."""
    n = int(g["n_views"])
    views = (ViewC * n)()
    keep = []
    for i in range(n):
        luma = np.ascontiguousarray(g[f"luma{i}"], np.float32)
        pts = np.ascontiguousarray(g[f"warp_points{i}"], np.float32)
        conf = np.ascontiguousarray(g[f"warp_confidence{i}"], np.float32)
        keep += [luma, pts, conf]
        v = views[i]
        v.luminance = fptr(luma)
        v.luma_height, v.luma_width = luma.shape
        v.width, v.height, v.has_camera, v.accepted = (int(x) for x in g[f"view{i}"])
        v.camera = CameraC.from_buffer_copy(g[f"camera{i}"].tobytes())
        v.warp.step, v.warp.columns, v.warp.rows = (int(x) for x in g[f"warp_shape{i}"])
        v.warp.points = fptr(pts)
        v.warp.confidence = fptr(conf)
        v.warp.capacity = int(v.warp.columns * v.warp.rows)
    return views, keep


def options_of(g: dict) -> DepthOptionsC:
    return DepthOptionsC.from_buffer_copy(g["options"].tobytes())


def run(g: dict, refine, extra=()) -> dict:
    """Call a refine_multiview_depth-shaped C function (the library's or the oracle's) on a
    fixture and collect the same outputs the fixture stores."""
    from oracle import oracle
    n = int(g["n_views"])
    views, keep = views_of(g)
    opt = options_of(g)
    m = int(g["fine_nodes"])
    refined = (WarpC * n)()
    pts = [np.full(2 * m, np.nan, np.float32) for _ in range(n)]
    conf = [np.full(m, np.nan, np.float32) for _ in range(n)]
    for i in range(n):
        refined[i].points = fptr(pts[i])
        refined[i].confidence = fptr(conf[i])
        refined[i].capacity = m
    reports = (DepthReportC * n)()
    out = {"depth": np.empty(m, np.float64), "confidence": np.empty(m, np.float32),
           "provenance": np.empty(m, np.uint8)}
    dmap = DepthMapC(capacity=m, depth=dptr(out["depth"]), confidence=fptr(out["confidence"]),
                     provenance=u8ptr(out["provenance"]))
    dbg_arrays = oracle.debug_buffers(n, int(g["coarse_nodes"]), int(g["labels"]), m)
    dbg = oracle.make_debug(dbg_arrays)
    status = refine(views, n, int(g["reference_index"]), C.byref(opt), refined, reports, C.byref(dmap),
                    C.byref(dbg), *extra)
    assert status == abi.OK, status
    for i in range(n):
        out[f"points{i}"] = pts[i]
        out[f"refined_confidence{i}"] = conf[i]
        r = reports[i]
        out[f"report{i}"] = np.array([float(getattr(r, f)) for f in REPORT_FIELDS], np.float64)
    for k in DEBUG_FIELDS:
        out[k] = dbg_arrays[k]
    return out


def compare(got: dict, g: dict):
    """Bitwise equality of every stored output (NaN patterns included)."""
    for k, v in got.items():
        want = g[k]
        assert want.dtype == v.dtype and want.shape == v.shape, k
        if v.dtype.kind == "f":
            bits = {4: np.uint32, 8: np.uint64}[v.dtype.itemsize]
            assert np.array_equal(v.view(bits), want.view(bits)), k
        else:
            assert np.array_equal(v, want), k
