"""ctypes wrapper of the CPU oracle (test infrastructure only).

Loads ``oracle/_build/libchiaro_oracle.so`` (built by ``make -C oracle``) and
exposes the restated reference functions to the tests, the smoke check and the
benchmark's CPU-baseline leg. Nothing in the ``chiaro_b200`` package imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from chiaro_b200 import abi
from chiaro_b200.abi import (CameraC, DepthDebugC, DepthMapC, DepthOptionsC, DepthReportC, ViewC, WarpC,
                             dptr, fptr, sizeptr, u8ptr, u16ptr)

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libchiaro_oracle.so"


def build(force: bool = False) -> Path:
    src = [HERE / "chiaro_oracle.cpp", HERE.parent / "include" / "chiaro_depth.h"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        P = C.POINTER
        sig = {
            "oracle_options_default": (None, [P(DepthOptionsC)]),
            "oracle_options_valid": (C.c_int, [P(DepthOptionsC)]),
            "oracle_refine_multiview_depth": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                                        P(WarpC), P(DepthReportC), P(DepthMapC), P(DepthDebugC),
                                                        C.c_int]),
            "oracle_inverse_depth_samples": (None, [C.c_double, C.c_double, C.c_size_t, P(C.c_double)]),
            "oracle_sublabel_depth": (C.c_double, [P(C.c_double), C.c_size_t, P(C.c_float), C.c_size_t]),
            "oracle_aggregate": (C.c_int, [P(C.c_float), C.c_size_t, P(DepthOptionsC), P(C.c_float)]),
            "oracle_semi_global_costs": (None, [P(C.c_float), P(C.c_float), C.c_size_t, C.c_size_t, C.c_size_t,
                                                P(C.c_float)]),
            "oracle_diagonal_paths": (C.c_size_t, [C.c_size_t, C.c_size_t, C.c_int, P(C.c_size_t),
                                                   P(C.c_size_t)]),
            "oracle_select_depths": (None, [P(C.c_double), C.c_size_t, P(C.c_float), P(C.c_float), P(C.c_uint8),
                                            C.c_size_t, P(DepthOptionsC), P(C.c_uint8), P(C.c_double),
                                            P(C.c_float), P(C.c_float), P(C.c_uint8), P(C.c_uint8)]),
            "oracle_complete_depth_field": (None, [P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                                   P(C.c_uint8), P(C.c_float), P(C.c_uint8), C.c_size_t,
                                                   C.c_size_t, P(DepthOptionsC)]),
            "oracle_reject_isolated": (None, [P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                              C.c_size_t, C.c_size_t, C.c_double]),
            "oracle_reject_small_components": (None, [P(C.c_uint8), P(C.c_double), P(C.c_float), C.c_size_t,
                                                      C.c_size_t, C.c_double, C.c_size_t]),
            "oracle_fit_local_planes": (None, [P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                               C.c_size_t, C.c_size_t, C.c_double]),
            "oracle_select_direct_depth": (C.c_int, [P(C.c_double), P(C.c_float), C.c_size_t, C.c_int, C.c_float,
                                                     C.c_int, P(DepthOptionsC), P(C.c_double), P(C.c_float),
                                                     P(C.c_float)]),
            "oracle_best_depth_candidate": (C.c_long, [P(C.c_double), P(C.c_float), C.c_size_t,
                                                       P(DepthOptionsC)]),
            "oracle_warp_decisions_agree": (C.c_int, [C.c_int, C.c_int, P(C.c_float), P(C.c_float), C.c_int,
                                                      P(C.c_float), P(C.c_float)]),
            "oracle_warp_decisions_filter": (None, [P(C.c_uint8), P(C.c_float), P(C.c_float), P(C.c_uint8),
                                                    P(C.c_float), C.c_size_t, C.c_size_t, C.c_int, C.c_int]),
            "oracle_diagnostic_samples": (None, [P(DepthMapC), P(C.c_uint16), P(C.c_uint16)]),
            "oracle_visualization_samples": (None, [P(DepthMapC), P(C.c_uint16)]),
            "oracle_distort": (None, [P(CameraC), P(C.c_double), P(C.c_double)]),
            "oracle_undistort": (None, [P(CameraC), P(C.c_double), P(C.c_double)]),
            "oracle_pixel_to_ray": (None, [P(CameraC), P(C.c_double), P(C.c_double), P(C.c_double)]),
            "oracle_project": (C.c_int, [P(CameraC), P(C.c_double), P(C.c_double)]),
            "oracle_map_from": (C.c_int, [P(CameraC), P(CameraC), P(C.c_double), C.c_double, P(C.c_double)]),
            "oracle_warp_map": (C.c_int, [P(WarpC), C.c_float, C.c_float, P(C.c_float)]),
            "oracle_warp_magnification": (C.c_int, [P(WarpC), C.c_float, C.c_float, P(C.c_float)]),
            "oracle_fit_homography_ransac": (C.c_int, [P(C.c_double), P(C.c_float), C.c_size_t, C.c_float,
                                                       P(C.c_double), P(C.c_size_t), P(C.c_float)]),
            "oracle_align_module": (C.c_int, [P(abi.AlignInputC), P(abi.AlignInputC), C.c_int,
                                              P(abi.AlignOptionsC), P(WarpC), P(WarpC), P(C.c_float),
                                              P(abi.AlignmentReportC), C.c_char_p]),
            "oracle_warp_confidence": (C.c_float, [P(WarpC), C.c_float, C.c_float]),
            "oracle_sample_nearest": (C.c_long, [P(DepthMapC), C.c_float, C.c_float]),
            "oracle_match_patch": (C.c_int, [P(C.c_float), C.c_size_t, C.c_size_t, P(C.c_float), C.c_size_t,
                                             C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                             P(C.c_float), P(C.c_float)]),
            "oracle_refine_resolution_warp": (C.c_int, [P(C.c_float), C.c_size_t, C.c_size_t, P(C.c_float),
                                                        C.c_size_t, C.c_size_t, P(WarpC), C.c_size_t, C.c_size_t,
                                                        P(WarpC), P(C.c_float)]),
            "oracle_plane_sample": (C.c_float, [P(C.c_float), C.c_size_t, C.c_size_t, C.c_float, C.c_float,
                                                P(C.c_int)]),
            "oracle_score_one_view": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, C.c_size_t, C.c_double,
                                                C.c_double, C.c_double, C.c_size_t, P(C.c_float)]),
            "oracle_build_cost_volume": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC), C.c_size_t,
                                                   C.c_size_t, P(C.c_float), P(C.c_float), P(C.c_float),
                                                   P(C.c_uint8), C.c_int]),
            "oracle_measure_direct_depths": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                                       P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_float),
                                                       P(C.c_uint8), C.c_size_t, C.c_size_t, P(C.c_uint8),
                                                       P(C.c_double), P(C.c_float), P(C.c_float), P(C.c_float),
                                                       P(C.c_uint8), C.c_int]),
            "oracle_target_decisions": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, C.c_size_t, P(DepthOptionsC),
                                                  P(C.c_uint8), P(C.c_double), P(C.c_float), P(C.c_uint8),
                                                  P(C.c_float), C.c_size_t, C.c_size_t, P(C.c_uint8)]),
            "oracle_luminance_half": (None, [P(C.c_uint16), C.c_size_t, C.c_size_t, C.c_float, C.c_float,
                                             P(C.c_float)]),
            "oracle_sgm_banded": (C.c_int, [P(C.c_float), P(C.c_float), C.c_size_t, C.c_size_t, C.c_size_t,
                                             P(C.c_int), C.c_size_t, C.c_size_t, C.c_size_t, P(C.c_int),
                                             P(C.c_uint8)]),
            "oracle_bandnet_features": (None, [P(C.c_float), P(C.c_float), C.c_size_t, C.c_size_t, C.c_size_t,
                                               P(C.c_float)]),
            "oracle_net_sample_labels": (None, [C.c_size_t, P(C.c_int)]),
            "oracle_bandnet_loss_grad_mode": (None, [P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_uint8),
                                                     C.c_size_t, C.c_size_t, C.c_size_t, P(C.c_float), P(C.c_float),
                                                     P(C.c_float), C.c_int]),
            "oracle_bandnet_loss_grad": (None, [P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_uint8), C.c_size_t,
                                                C.c_size_t, C.c_size_t, P(C.c_float), P(C.c_float), P(C.c_float)]),
            "oracle_sgm_u16": (None, [P(C.c_float), P(C.c_float), C.c_size_t, C.c_size_t, C.c_size_t,
                                      P(C.c_uint16), P(C.c_uint16)]),
            "oracle_stage_sample": (C.c_int, [P(ViewC), C.c_size_t, C.c_size_t, P(DepthOptionsC), P(C.c_uint8),
                                              C.c_int, P(C.c_double), P(C.c_uint64)]),
            "oracle_luminance_half_mesh": (None, [P(C.c_uint16), C.c_size_t, C.c_size_t, C.c_float, C.c_float,
                                                  P(C.c_float), C.c_size_t, C.c_size_t, P(C.c_float),
                                                  P(C.c_float)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def default_options() -> DepthOptionsC:
    o = DepthOptionsC()
    lib().oracle_options_default(C.byref(o))
    return o


def refine_multiview_depth(inputs, reference_index, alignments, options, threads: int = 0, debug=None):
    """Run the oracle's whole stage; returns a dict of numpy outputs or None."""
    from chiaro_b200.depth import output_shape, pack_views

    n = len(inputs)
    ref = inputs[reference_index]
    (columns, rows, step), (cc, cr, cs) = output_shape(ref.width, ref.height, options)
    m = columns * rows
    views, keep = pack_views(inputs, alignments)
    refined = (WarpC * n)()
    pts = [np.full(2 * m, np.nan, dtype=np.float32) for _ in range(n)]
    conf = [np.full(m, np.nan, dtype=np.float32) for _ in range(n)]
    for i in range(n):
        refined[i].points = fptr(pts[i])
        refined[i].confidence = fptr(conf[i])
        refined[i].capacity = m
    reports = (DepthReportC * n)()
    depth = np.empty(m, dtype=np.float64)
    confidence = np.empty(m, dtype=np.float32)
    provenance = np.empty(m, dtype=np.uint8)
    dmap = DepthMapC()
    dmap.capacity = m
    dmap.depth = dptr(depth)
    dmap.confidence = fptr(confidence)
    dmap.provenance = u8ptr(provenance)
    dbg = None
    if debug is not None:
        dbg = make_debug(debug)
    opt = options.to_c()
    status = lib().oracle_refine_multiview_depth(views, n, reference_index, C.byref(opt), refined, reports,
                                                 C.byref(dmap), C.byref(dbg) if dbg is not None else None, threads)
    if status == abi.INVALID:
        return None
    assert status == abi.OK, status
    return dict(columns=int(dmap.columns), rows=int(dmap.rows), step=int(dmap.step), depth=depth,
                confidence=confidence, provenance=provenance, points=pts, warp_confidence=conf,
                reports=[reports[i] for i in range(n)], refined=[refined[i] for i in range(n)])


def make_debug(arrays: dict) -> DepthDebugC:
    dbg = DepthDebugC()
    for name, arr in arrays.items():
        ctype = abi.DEBUG_FIELD_TYPES[name]
        setattr(dbg, name, arr.ctypes.data_as(C.POINTER(ctype)))
    return dbg


def debug_buffers(n_views: int, coarse_nodes: int, labels: int, fine_nodes: int) -> dict:
    """Allocate every debug field with its documented size."""
    N, D, M = coarse_nodes, labels, fine_nodes
    f32, f64, u8 = np.float32, np.float64, np.uint8
    spec = dict(coarse_scores=(N * D, f32), coarse_costs=(N * D, f32), coarse_guidance=(N, f32),
                coarse_tested=(N, u8), regularised=(N * D, f32), coarse_has=(N, u8), coarse_depth=(N, f64),
                coarse_confidence=(N, f32), coarse_improvement=(N, f32), coarse_regularized=(N, u8),
                coarse_fillable=(N, u8), direct_has=(M, u8), direct_depth=(M, f64), direct_confidence=(M, f32),
                direct_improvement=(M, f32), direct_regularized=(M, u8), direct_guidance=(M, f32),
                direct_tested=(M, u8), isolated_has=(M, u8), component_has=(M, u8), fitted_depth=(M, f64),
                decision_kind=(n_views * M, u8))
    return {k: np.zeros(n, dtype=t) for k, (n, t) in spec.items()}


def semi_global_costs(costs: np.ndarray, guidance: np.ndarray, columns: int, rows: int, labels: int) -> np.ndarray:
    out = np.empty(columns * rows * labels, dtype=np.float32)
    costs = np.ascontiguousarray(costs, dtype=np.float32)
    guidance = np.ascontiguousarray(guidance, dtype=np.float32)
    lib().oracle_semi_global_costs(fptr(costs), fptr(guidance), columns, rows, labels, fptr(out))
    return out


def threads_default() -> int:
    return os.cpu_count() or 1


def refine_resolution_warp(reference, target, base, width: int, height: int):
    """oracle_refine_resolution_warp (resolution.rs:232-439) on chiaro_b200's Plane and Warp
    types; returns a chiaro_b200.resolution.ResolutionWarp."""
    from chiaro_b200.align import Warp
    from chiaro_b200.resolution import WARP_STEP, ResolutionAlignmentReport, ResolutionWarp, warp_c
    F = C.POINTER(C.c_float)
    columns, rows = -(-width // WARP_STEP) + 1, -(-height // WARP_STEP) + 1
    points = np.empty((columns * rows, 2), np.float32)
    confidence = np.empty(columns * rows, np.float32)
    out = WarpC(capacity=columns * rows, points=points.ctypes.data_as(F), confidence=confidence.ctypes.data_as(F))
    report = np.zeros(4, np.float32)
    ref = np.ascontiguousarray(reference.data, np.float32)
    tgt = np.ascontiguousarray(target.data, np.float32)
    base_c = warp_c(base)
    st = lib().oracle_refine_resolution_warp(ref.ctypes.data_as(F), reference.width, reference.height,
                                             tgt.ctypes.data_as(F), target.width, target.height, C.byref(base_c),
                                             width, height, C.byref(out), report.ctypes.data_as(F))
    assert st == 0, st
    return ResolutionWarp(Warp(WARP_STEP, columns, rows, points, confidence),
                          ResolutionAlignmentReport(*[float(v) for v in report]))


def align_module(reference, target, options=None, seed=None):
    """oracle_align_module (align.rs:281-519) on chiaro_b200's AlignInput types:
    (warp points [n, 2], confidence [n], gain, chiaro_alignment_report)."""
    from chiaro_b200.align import AlignOptions, align_input_c
    F = C.POINTER(C.c_float)
    options = options or AlignOptions()
    ref_c, keep_r = align_input_c(reference)
    tgt_c, keep_t = align_input_c(target)
    step = options.grid_step
    columns, rows = -(-reference.width // step) + 1, -(-reference.height // step) + 1
    points = np.empty((columns * rows, 2), np.float32)
    confidence = np.empty(columns * rows, np.float32)
    out = WarpC(capacity=columns * rows, points=points.ctypes.data_as(F), confidence=confidence.ctypes.data_as(F))
    seed_c, keep_s = None, None
    if seed is not None:
        keep_s = (np.ascontiguousarray(seed.points, np.float32), np.ascontiguousarray(seed.confidence, np.float32))
        seed_c = WarpC(step=seed.step, columns=seed.columns, rows=seed.rows, points=keep_s[0].ctypes.data_as(F),
                       confidence=keep_s[1].ctypes.data_as(F), capacity=seed.columns * seed.rows)
    gain = C.c_float()
    report = abi.AlignmentReportC()
    opt = options.to_c()
    st = lib().oracle_align_module(C.byref(ref_c), C.byref(tgt_c), int(reference.name == target.name), C.byref(opt),
                                   C.byref(seed_c) if seed_c is not None else None, C.byref(out), C.byref(gain),
                                   C.byref(report), None)
    assert st == 0, st
    return points, confidence, gain.value, report
