"""Shared cases of the resolution-warp tests: the reference's own test signals
(resolution.rs:532-562, image.rs:645-668) and the oracle's refine_resolution_warp."""
import ctypes as C

import numpy as np

from chiaro_b200.align import Warp
from chiaro_b200.image import Plane
from chiaro_b200.resolution import warp_c

F = C.POINTER(C.c_float)


def kat_signal(x, y):
    """resolution.rs:533-537, in f32."""
    x, y = np.float32(x), np.float32(y)
    return (np.sin(x * np.float32(0.27)) * np.cos(y * np.float32(0.19))
            + np.float32(0.35) * np.sin(x * np.float32(0.073) + y * np.float32(0.11))
            + np.float32(0.12) * np.cos(x * np.float32(0.41) - y * np.float32(0.037))).astype(np.float32)


def textured(width, height, shift):
    """image.rs:645-655, in f32."""
    y, x = np.mgrid[0:height, 0:width].astype(np.float32)
    fx, fy = x - np.float32(shift[0]), y - np.float32(shift[1])
    return (np.sin(fx * np.float32(0.31)) * np.cos(fy * np.float32(0.17))
            + np.float32(0.3) * np.sin(fx * np.float32(0.05) + fy * np.float32(0.07))).astype(np.float32)


def identity_warp(width, height, step=32, scale=1.0, offset=(0.0, 0.0), undefined=None):
    """Warp::from_fn (align.rs:50-80) of q = scale * p + offset; `undefined(p)` marks None nodes."""
    columns, rows = -(-width // step) + 1, -(-height // step) + 1
    r, c = np.divmod(np.arange(columns * rows), columns)
    px, py = (c * step).astype(np.float64), (r * step).astype(np.float64)
    points = np.stack([scale * px + offset[0], scale * py + offset[1]], axis=1).astype(np.float32)
    confidence = np.ones(columns * rows, np.float32)
    if undefined is not None:
        none = undefined(px, py)
        points[none] = np.nan
        confidence[none] = 0.0
    return Warp(step, columns, rows, points, confidence)


def kat_planes(shift=(0.6, -0.35), size=(256, 192)):
    w, h = size
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    reference = Plane(w, h, kat_signal(x, y))
    target = Plane(w, h, kat_signal(x - np.float32(shift[0]), y - np.float32(shift[1])))
    return reference, target


def oracle_refine(lib, reference, target, base, width, height):
    from oracle import oracle
    return oracle.refine_resolution_warp(reference, target, base, width, height)


def warp_map(warp, x, y):
    """Warp::map through the oracle (align.rs:84-111)."""
    from oracle import oracle
    out = np.zeros(2, np.float32)
    wc = warp_c(warp)
    ok = oracle.lib().oracle_warp_map(C.byref(wc), x, y, out.ctypes.data_as(F))
    return out if ok else None
