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
class LevelReport:
    """align.rs:202-207."""

    scale: int
    patches: int
    inliers: int
    median_residual_px: float


@dataclass
class AlignmentReport:
    """AlignmentReport (align.rs:160-200) without the focus fields (other stages fill them)."""

    camera: str = ""
    accepted: bool = True
    depth: Optional[object] = None  # DepthAlignmentReport once the depth stage ran
    status: str = ""
    initialised_from: str = ""
    coverage: float = 0.0
    correction_median_px: tuple = (0.0, 0.0)
    levels: list = field(default_factory=list)
    inliers: int = 0
    patches: int = 0
    residual_median_px: float = 0.0
    residual_p90_px: float = 0.0
    inlier_ratio: float = 0.0


@dataclass
class AlignOptions:
    """AlignOptions (align.rs:205-243) without the depth options."""

    grid_step: int = 32
    patch: int = 32
    coarse_radius: int = 12
    min_score: float = 0.5
    inlier_px: float = 3.0
    min_inlier_ratio: float = 0.45
    refine: bool = True

    def to_c(self):
        from .abi import AlignOptionsC
        return AlignOptionsC(grid_step=self.grid_step, patch=self.patch, coarse_radius=self.coarse_radius,
                             min_score=self.min_score, inlier_px=self.inlier_px,
                             min_inlier_ratio=self.min_inlier_ratio, refine=1 if self.refine else 0)


@dataclass
class ModuleAlignment:
    """align.rs:148-157."""

    name: str
    warp: Warp
    gain: float = 1.0
    offset: float = 0.0
    report: AlignmentReport = field(default_factory=AlignmentReport)


def align_input_c(inp: AlignInput):
    """(chiaro_align_input, keepalive) of an AlignInput."""
    import ctypes as C

    from .abi import AlignInputC
    luma = np.ascontiguousarray(inp.luminance.data, dtype=np.float32)
    c = AlignInputC(luminance=luma.ctypes.data_as(C.POINTER(C.c_float)), luma_width=inp.luminance.width,
                    luma_height=inp.luminance.height, width=inp.width, height=inp.height,
                    has_camera=1 if inp.camera is not None else 0, nominal_focal_px=float(inp.nominal_focal_px))
    if inp.camera is not None:
        c.camera = inp.camera.to_c()
    return c, luma


def report_from_c(r, camera: str, seed_name: str = "seed") -> AlignmentReport:
    """An AlignmentReport from the library's chiaro_alignment_report, the status text as align.rs:465-477 writes it."""
    from .abi import ALIGN_STATUS, INITIALISED_FROM
    status = ALIGN_STATUS[r.status]
    if r.status == 1:
        status = f"rejected: {r.inlier_ratio * 100.0:.0f}% correspondence consensus"
    initialised = INITIALISED_FROM[r.initialised_from] or seed_name
    levels = [LevelReport(int(lv.scale), int(lv.patches), int(lv.inliers), float(lv.median_residual_px))
              for lv in r.levels[:r.n_levels]]
    return AlignmentReport(camera=camera, accepted=bool(r.accepted), status=status, initialised_from=initialised,
                           coverage=float(r.coverage),
                           correction_median_px=(float(r.correction_median_px[0]), float(r.correction_median_px[1])),
                           levels=levels, inliers=int(r.inliers), patches=int(r.patches),
                           residual_median_px=float(r.residual_median_px), residual_p90_px=float(r.residual_p90_px),
                           inlier_ratio=float(r.inlier_ratio))


class AlignmentError(RuntimeError):
    """align_module's Err (the no-calibration search found no correlation)."""


def align_module(reference: AlignInput, target: AlignInput, options: Optional[AlignOptions] = None,
                 seed: Optional[Warp] = None, seed_name: str = "seed", context=None) -> ModuleAlignment:
    """align_module / align_module_seeded (align.rs:272-519) on the GPU (chiaro_align_module):
    the target's warp from the reference raster, its photometric gain and report. Raises
    AlignmentError where the reference returns Err."""
    import ctypes as C

    from .abi import INVALID, AlignmentReportC, WarpC
    from .runtime import default_context
    ctx = context or default_context()
    options = options or AlignOptions()
    ref_c, keep_r = align_input_c(reference)
    tgt_c, keep_t = align_input_c(target)
    step = options.grid_step
    columns, rows = -(-reference.width // step) + 1, -(-reference.height // step) + 1
    points = np.empty((columns * rows, 2), np.float32)
    confidence = np.empty(columns * rows, np.float32)
    F = C.POINTER(C.c_float)
    out = WarpC(capacity=columns * rows, points=points.ctypes.data_as(F), confidence=confidence.ctypes.data_as(F))
    seed_c = None
    if seed is not None:
        seed_points = np.ascontiguousarray(seed.points, np.float32)
        seed_conf = np.ascontiguousarray(seed.confidence, np.float32)
        seed_c = WarpC(step=seed.step, columns=seed.columns, rows=seed.rows, points=seed_points.ctypes.data_as(F),
                       confidence=seed_conf.ctypes.data_as(F), capacity=seed.columns * seed.rows)
    gain = C.c_float()
    report = AlignmentReportC()
    opt = options.to_c()
    st = ctx.lib.chiaro_align_module(ctx.handle, C.byref(ref_c), C.byref(tgt_c), int(reference.name == target.name),
                                     C.byref(opt), C.byref(seed_c) if seed_c is not None else None, C.byref(out),
                                     C.byref(gain), C.byref(report))
    if st == INVALID:
        raise AlignmentError(ctx.lib.chiaro_depth_last_error(ctx.handle).decode())
    ctx.check(st)
    return ModuleAlignment(name=target.name, warp=Warp(step, columns, rows, points, confidence), gain=float(gain.value),
                           offset=0.0, report=report_from_c(report, target.name, seed_name))
