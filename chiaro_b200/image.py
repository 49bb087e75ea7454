"""Image containers: ``Plane`` (crates/chiaro-fusion/src/image.rs:431-514) and the
part of ``Mosaic`` (image.rs:16-35) the depth stage's input needs.

``Plane.sample`` is the bilinear texel fetch of image.rs:451-466, written with
numpy float32 scalars so it rounds as the Rust code does. The depth kernels
carry their own device copy of it. ``Mosaic.luminance_half`` (image.rs:401-428)
runs on the GPU (``chiaro_luminance_half``); there is no host fallback.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import ctypes as C

import numpy as np


@dataclass
class Plane:
    """Single-channel f32 image, row-major ``data[y * width + x]``."""

    width: int
    height: int
    data: np.ndarray

    def __post_init__(self):
        self.data = np.ascontiguousarray(self.data, dtype=np.float32).reshape(self.height, self.width)

    def at(self, x: int, y: int) -> np.float32:
        return self.data[y, x]

    def sample(self, x, y) -> Optional[np.float32]:
        """image.rs:451-466; None outside [0, w-1] x [0, h-1]."""
        x = np.float32(x)
        y = np.float32(y)
        if not (x >= 0 and y >= 0 and x <= np.float32(self.width - 1) and y <= np.float32(self.height - 1)):
            return None
        x0 = int(np.floor(x))
        y0 = int(np.floor(y))
        x1 = min(x0 + 1, self.width - 1)
        y1 = min(y0 + 1, self.height - 1)
        one = np.float32(1.0)
        tx = x - np.float32(x0)
        ty = y - np.float32(y0)
        top = self.at(x0, y0) * (one - tx) + self.at(x1, y0) * tx
        bottom = self.at(x0, y1) * (one - tx) + self.at(x1, y1) * tx
        return np.float32(top * (one - ty) + bottom * ty)


@dataclass
class VignettingMesh:
    """Flat-field gains over the sensor raster (calibration.rs:354-380), row-major [rows][columns]."""

    columns: int
    rows: int
    gains: np.ndarray

    def __post_init__(self):
        self.gains = np.ascontiguousarray(self.gains, dtype=np.float32).reshape(-1)
        assert self.gains.size == self.columns * self.rows


@dataclass
class Mosaic:
    """A module's raw mosaic in the calibration raster: u16 Q6 samples (RAW code << 6),
    black and white levels in Q6 units, the optional flat-field mesh (image.rs:16-35)."""

    width: int
    height: int
    samples: np.ndarray
    black_q6: float
    white_q6: float
    vignetting: Optional[VignettingMesh] = None

    def __post_init__(self):
        self.samples = np.ascontiguousarray(self.samples, dtype=np.uint16).reshape(self.height, self.width)

    def luminance_half(self, context=None) -> Plane:
        """Half-resolution log-luminance plane (image.rs:401-428), computed on the GPU: the
        2x2 mean, black/white scaling and flat field are the reference's f32 arithmetic;
        the log is correctly rounded, within 1 ulp of the host logf the reference uses."""
        from . import abi, runtime
        ctx = context or runtime.default_context()
        out = np.empty((self.height // 2) * (self.width // 2), np.float32)
        mesh = None
        if self.vignetting is not None:
            mesh = abi.VignettingC(columns=self.vignetting.columns, rows=self.vignetting.rows,
                                   gains=self.vignetting.gains.ctypes.data_as(C.POINTER(C.c_float)))
        ctx.check(ctx.lib.chiaro_luminance_half(
            ctx.handle, self.samples.ctypes.data_as(C.POINTER(C.c_uint16)), self.width, self.height,
            float(self.black_q6), float(self.white_q6), C.byref(mesh) if mesh is not None else None,
            out.ctypes.data_as(C.POINTER(C.c_float))))
        return Plane(self.width // 2, self.height // 2, out)
