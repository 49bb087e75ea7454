"""Alignment types consumed and produced by the depth stage.

Mirrors ``Warp``, ``AlignInput``, ``ModuleAlignment`` and ``AlignmentReport``
(crates/chiaro-fusion/src/align.rs:34-257). ``Warp.map`` is the bilinear grid
lookup of align.rs:84-111 in numpy float32, vectorised over points.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from .camera import ResolvedCamera
from .image import Plane

FAR_DEPTH = 1.0e8  # align.rs:266, depth used for the rotation-only initialisation


@dataclass
class Warp:
    """Reference-raster pixel -> module-raster pixel on a ``step`` grid.

    ``points`` has shape (rows*columns, 2) float32 with NaN where undefined;
    ``confidence`` has shape (rows*columns,).
    """

    step: int
    columns: int
    rows: int
    points: np.ndarray
    confidence: np.ndarray

    def __post_init__(self):
        self.points = np.ascontiguousarray(self.points, dtype=np.float32).reshape(self.rows * self.columns, 2)
        self.confidence = np.ascontiguousarray(self.confidence, dtype=np.float32).reshape(self.rows * self.columns)

    @staticmethod
    def from_fn(width: int, height: int, step: int,
                fn: Callable[[np.ndarray], tuple]) -> "Warp":
        """align.rs:50-82. ``fn`` takes an (n, 2) f64 array of grid pixels and
        returns (q[n, 2] f64, valid[n] bool)."""
        columns = -(-width // step) + 1
        rows = -(-height // step) + 1
        r, c = np.meshgrid(np.arange(rows), np.arange(columns), indexing="ij")
        p = np.stack([(c * step).astype(np.float64), (r * step).astype(np.float64)], -1).reshape(-1, 2)
        q, valid = fn(p)
        valid = np.asarray(valid, dtype=bool)
        points = np.where(valid[:, None], np.asarray(q, dtype=np.float64).astype(np.float32), np.float32(np.nan))
        confidence = np.where(valid, np.float32(1.0), np.float32(0.0)).astype(np.float32)
        return Warp(step, columns, rows, points, confidence)

    @staticmethod
    def identity(width: int, height: int, step: int) -> "Warp":
        return Warp.from_fn(width, height, step, lambda p: (p, np.ones(len(p), dtype=bool)))

    @staticmethod
    def calibrated(reference: ResolvedCamera, target: ResolvedCamera, width: int, height: int,
                   step: int, depth: float = FAR_DEPTH) -> "Warp":
        """The calibrated infinity mapping of align.rs:317-324 on a ``step`` grid."""
        def fn(p):
            q, valid = target.map_from(reference, p, depth)
            return q, valid & np.isfinite(q).all(axis=-1)
        return Warp.from_fn(width, height, step, fn)

    def map(self, x, y):
        """align.rs:84-111, vectorised. Returns (q[..., 2] float32, valid[...])."""
        x = np.asarray(x, dtype=np.float32)
        y = np.asarray(y, dtype=np.float32)
        one = np.float32(1.0)
        fx = x / np.float32(self.step)
        fy = y / np.float32(self.step)
        ok = ~((fx < 0) | (fy < 0))
        with np.errstate(invalid="ignore"):
            c0 = np.minimum(_sat(np.floor(fx)), self.columns - 1)
            r0 = np.minimum(_sat(np.floor(fy)), self.rows - 1)
        c1 = np.minimum(c0 + 1, self.columns - 1)
        r1 = np.minimum(r0 + 1, self.rows - 1)
        tx = fx - c0.astype(np.float32)
        ty = fy - r0.astype(np.float32)
        pts = self.points.reshape(self.rows, self.columns, 2)
        a, b, c, d = pts[r0, c0], pts[r0, c1], pts[r1, c0], pts[r1, c1]
        txe, tye = tx[..., None], ty[..., None]
        top = a * (one - txe) + b * txe
        bottom = c * (one - txe) + d * txe
        out = (top * (one - tye) + bottom * tye).astype(np.float32)
        ok = ok & ~np.isnan(out).any(axis=-1)
        return out, ok

    def confidence_at(self, x, y):
        """align.rs:113-131: bilinear confidence clamped to [0, 1]."""
        x = np.asarray(x, dtype=np.float32)
        y = np.asarray(y, dtype=np.float32)
        one = np.float32(1.0)
        fx = x / np.float32(self.step)
        fy = y / np.float32(self.step)
        c0 = np.minimum(_sat(np.floor(fx)), self.columns - 1)
        r0 = np.minimum(_sat(np.floor(fy)), self.rows - 1)
        c1 = np.minimum(c0 + 1, self.columns - 1)
        r1 = np.minimum(r0 + 1, self.rows - 1)
        tx = fx - c0.astype(np.float32)
        ty = fy - r0.astype(np.float32)
        conf = self.confidence.reshape(self.rows, self.columns)
        top = conf[r0, c0] * (one - tx) + conf[r0, c1] * tx
        bottom = conf[r1, c0] * (one - tx) + conf[r1, c1] * tx
        out = np.clip(top * (one - ty) + bottom * ty, np.float32(0), np.float32(1)).astype(np.float32)
        return np.where((fx < 0) | (fy < 0), np.float32(0), out)


def _sat(v: np.ndarray) -> np.ndarray:
    """Rust `as usize` for non-negative floats: NaN -> 0, saturating."""
    v = np.nan_to_num(np.asarray(v, dtype=np.float64), nan=0.0, posinf=2.0 ** 62, neginf=0.0)
    return np.clip(v, 0, 2.0 ** 62).astype(np.int64)


@dataclass
class AlignInput:
    """One module's inputs (align.rs:246-257)."""

    name: str
    luminance: Plane
    width: int
    height: int
    camera: Optional[ResolvedCamera]
    nominal_focal_px: float = 0.0


@dataclass
class AlignmentReport:
    """The fields of AlignmentReport (align.rs:160-200) the depth stage reads and writes."""

    camera: str = ""
    accepted: bool = True
    depth: Optional[object] = None  # DepthAlignmentReport once the depth stage ran
    status: str = ""


@dataclass
class ModuleAlignment:
    """align.rs:148-157."""

    name: str
    warp: Warp
    gain: float = 1.0
    offset: float = 0.0
    report: AlignmentReport = field(default_factory=AlignmentReport)
