"""refine_resolution_warp (crates/chiaro-fusion/src/resolution.rs:232-439) on the GPU.

The target's half-resolution luminance is resampled into the reference plane through
the base warp and a 12 x 12 patch is matched around every node of a 32 px control
grid (``chiaro_refine_resolution_warp``: a render kernel and a warp-per-node patch
search; the grid's median filter and hole completion run in the library on the
host). The result is bit-identical to the reference's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
import numpy as np

from . import abi
from .align import Warp
from .image import Plane

WARP_STEP = 32  # LOCAL_WARP_STEP (resolution.rs:18)


@dataclass
class ResolutionAlignmentReport:
    """resolution.rs:88-100."""

    verified_fraction: float
    supported_fraction: float
    median_correction_px: float
    mean_confidence: float


@dataclass
class ResolutionWarp:
    """resolution.rs:102-105."""

    warp: Warp
    report: ResolutionAlignmentReport


def warp_c(warp: Warp) -> abi.WarpC:
    """A chiaro_warp view of a Warp's arrays (the Warp must outlive it)."""
    return abi.WarpC(step=warp.step, columns=warp.columns, rows=warp.rows,
                     points=warp.points.ctypes.data_as(C.POINTER(C.c_float)),
                     confidence=warp.confidence.ctypes.data_as(C.POINTER(C.c_float)),
                     capacity=warp.columns * warp.rows)


def refine_resolution_warp(reference: Plane, target: Plane, base: Warp, width: int, height: int,
                           context=None) -> ResolutionWarp:
    """The reference's refine_resolution_warp: ``reference`` and ``target`` are half-resolution
    luminance planes, ``base`` the target's warp from the ``width`` x ``height`` reference raster.
    A plane may also be given as a CUDA tensor (row-major f32 on the context's device); then
    both must be, and they are read in place."""
    from .runtime import default_context
    ctx = context or default_context()
    if not isinstance(reference, Plane):
        return _refine_device(reference, target, base, width, height, ctx)
    columns, rows = -(-width // WARP_STEP) + 1, -(-height // WARP_STEP) + 1
    points = np.empty((columns * rows, 2), np.float32)
    confidence = np.empty(columns * rows, np.float32)
    out = abi.WarpC(capacity=columns * rows, points=points.ctypes.data_as(C.POINTER(C.c_float)),
                    confidence=confidence.ctypes.data_as(C.POINTER(C.c_float)))
    report = abi.ResolutionReportC()
    ref = np.ascontiguousarray(reference.data, np.float32)
    tgt = np.ascontiguousarray(target.data, np.float32)
    base_c = warp_c(base)
    ctx.check(ctx.lib.chiaro_refine_resolution_warp(
        ctx.handle, ref.ctypes.data_as(C.POINTER(C.c_float)), reference.width, reference.height,
        tgt.ctypes.data_as(C.POINTER(C.c_float)), target.width, target.height, C.byref(base_c), width, height,
        C.byref(out), C.byref(report)))
    return ResolutionWarp(Warp(WARP_STEP, columns, rows, points, confidence),
                          ResolutionAlignmentReport(report.verified_fraction, report.supported_fraction,
                                                    report.median_correction_px, report.mean_confidence))



def _refine_device(reference, target, base: Warp, width: int, height: int, ctx) -> ResolutionWarp:
    """chiaro_refine_resolution_warp_device on two CUDA tensors of shape (height, width)."""
    columns, rows = -(-width // WARP_STEP) + 1, -(-height // WARP_STEP) + 1
    points = np.empty((columns * rows, 2), np.float32)
    confidence = np.empty(columns * rows, np.float32)
    out = abi.WarpC(capacity=columns * rows, points=points.ctypes.data_as(C.POINTER(C.c_float)),
                    confidence=confidence.ctypes.data_as(C.POINTER(C.c_float)))
    report = abi.ResolutionReportC()
    ref, tgt = reference.contiguous(), target.contiguous()
    base_c = warp_c(base)
    ctx.check(ctx.lib.chiaro_refine_resolution_warp_device(
        ctx.handle, ref.data_ptr(), ref.shape[1], ref.shape[0], tgt.data_ptr(), tgt.shape[1], tgt.shape[0],
        C.byref(base_c), width, height, C.byref(out), C.byref(report)))
    return ResolutionWarp(Warp(WARP_STEP, columns, rows, points, confidence),
                          ResolutionAlignmentReport(report.verified_fraction, report.supported_fraction,
                                                    report.median_correction_px, report.mean_confidence))
