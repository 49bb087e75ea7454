"""Host API of the depth stage: the Python form of ``chiaro_fusion::depth``.

``refine_multiview_depth(inputs, reference_index, alignments, options)``
keeps the signature and the semantics of the Rust function
(crates/chiaro-fusion/src/depth.rs:312-580): it returns ``None`` where the
reference returns ``None``, replaces ``alignments[t].warp`` and sets
``alignments[t].report.depth`` for every accepted calibrated target, and
returns the ``DenseDepthMap``. All of the work runs in the CUDA library
``libchiaro_depth.so`` through its C ABI; there is no CPU fallback, and the
call raises if the library cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import struct
import zlib
from dataclasses import dataclass, field
from enum import IntEnum
from pathlib import Path
from typing import Iterable, List, Optional, Sequence

import numpy as np

from . import abi
from .abi import DepthMapC, DepthOptionsC, DepthReportC, ViewC, WarpC, dptr, fptr, u8ptr


@dataclass
class DepthOptions:
    """DepthOptions with the reference defaults (depth.rs:39-91)."""

    enabled: bool = True
    grid_step: int = 8
    near_depth: float = 500.0
    far_depth: float = 10_000_000.0
    planes: int = 96
    patch_radius: int = 4
    minimum_support: int = 2
    best_view_count: int = 3
    minimum_score: float = 0.45
    minimum_margin: float = 0.01
    minimum_improvement: float = 0.01
    minimum_neighbour_support: int = 2
    completion_iterations: int = 0

    def to_c(self) -> DepthOptionsC:
        o = DepthOptionsC()
        o.enabled = 1 if self.enabled else 0
        o.grid_step = int(self.grid_step)
        o.near_depth = float(self.near_depth)
        o.far_depth = float(self.far_depth)
        o.planes = int(self.planes)
        o.patch_radius = int(self.patch_radius)
        o.minimum_support = int(self.minimum_support)
        o.best_view_count = int(self.best_view_count)
        o.minimum_score = float(self.minimum_score)
        o.minimum_margin = float(self.minimum_margin)
        o.minimum_improvement = float(self.minimum_improvement)
        o.minimum_neighbour_support = int(self.minimum_neighbour_support)
        o.completion_iterations = int(self.completion_iterations)
        return o

    def is_valid(self) -> bool:
        """valid_options (depth.rs:1879-1891)."""
        return (self.enabled and self.grid_step > 0 and np.isfinite(self.near_depth)
                and np.isfinite(self.far_depth) and self.near_depth > 0.0
                and self.far_depth > self.near_depth and self.planes >= 3 and self.patch_radius > 0
                and self.minimum_support > 0 and self.best_view_count >= self.minimum_support
                and self.minimum_neighbour_support > 0)


class DepthProvenance(IntEnum):
    """depth.rs:115-121."""

    Unsupported = abi.UNSUPPORTED
    Global = abi.GLOBAL
    Measured = abi.MEASURED
    Regularized = abi.REGULARIZED


@dataclass
class DenseDepthNode:
    """depth.rs:123-128."""

    depth: Optional[float]
    confidence: float
    provenance: DepthProvenance


@dataclass
class DepthAlignmentReport:
    """depth.rs:93-113."""

    tested_nodes: int = 0
    measured_nodes: int = 0
    regularized_nodes: int = 0
    fallback_nodes: int = 0
    refined_nodes: int = 0
    occluded_nodes: int = 0
    boundary_nodes: int = 0
    reconstructed_fraction: float = 0.0
    refined_fraction: float = 0.0
    occluded_fraction: float = 0.0
    median_depth: Optional[float] = None
    median_score_improvement: Optional[float] = None

    @staticmethod
    def from_c(r: DepthReportC) -> "DepthAlignmentReport":
        return DepthAlignmentReport(
            tested_nodes=r.tested_nodes, measured_nodes=r.measured_nodes,
            regularized_nodes=r.regularized_nodes, fallback_nodes=r.fallback_nodes,
            refined_nodes=r.refined_nodes, occluded_nodes=r.occluded_nodes,
            boundary_nodes=r.boundary_nodes,
            reconstructed_fraction=float(np.float32(r.reconstructed_fraction)),
            refined_fraction=float(np.float32(r.refined_fraction)),
            occluded_fraction=float(np.float32(r.occluded_fraction)),
            median_depth=float(r.median_depth) if r.has_median_depth else None,
            median_score_improvement=(float(np.float32(r.median_score_improvement))
                                      if r.has_median_score_improvement else None))


@dataclass
class DenseDepthMap:
    """depth.rs:133-141, stored as arrays: ``depth`` (NaN = None),
    ``confidence`` and ``provenance`` of ``columns * rows`` nodes."""

    columns: int
    rows: int
    step: int
    near_depth: float
    far_depth: float
    depth: np.ndarray
    confidence: np.ndarray
    provenance: np.ndarray

    @property
    def nodes(self) -> List[DenseDepthNode]:
        return [self._node(i) for i in range(self.columns * self.rows)]

    def _node(self, i: int) -> DenseDepthNode:
        d = float(self.depth[i])
        return DenseDepthNode(None if np.isnan(d) else d, float(self.confidence[i]),
                              DepthProvenance(int(self.provenance[i])))

    def node(self, column: int, row: int) -> Optional[DenseDepthNode]:
        """depth.rs:144-146."""
        if column < self.columns and row < self.rows:
            return self._node(row * self.columns + column)
        return None

    def sample_nearest(self, x: float, y: float) -> Optional[DenseDepthNode]:
        """depth.rs:152-159: nearest node, no interpolation."""
        if x < 0.0 or y < 0.0 or self.step == 0:
            return None
        column = int(_round_half_away(np.float32(x) / np.float32(self.step)))
        row = int(_round_half_away(np.float32(y) / np.float32(self.step)))
        return self.node(column, row)

    def diagnostic_samples(self):
        """depth.rs:200-222: (inverse-depth u16[n], provenance u16[3n])."""
        near_inverse = 1.0 / self.near_depth
        far_inverse = 1.0 / self.far_depth
        rng = max(near_inverse - far_inverse, np.finfo(np.float64).tiny)
        has = np.isin(self.provenance, (abi.MEASURED, abi.REGULARIZED))
        with np.errstate(divide="ignore", invalid="ignore"):
            normalized = np.clip((1.0 / self.depth - far_inverse) / rng, 0.0, 1.0)
        encoded = np.where(has, 1 + _round_u16(normalized * 65534.0).astype(np.int64), 0).astype(np.uint16)
        conf = np.clip(self.confidence.astype(np.float32), np.float32(0), np.float32(1))
        scale = (np.float32(0.35) + np.float32(0.65) * conf).astype(np.float64)
        color = np.zeros((len(self.provenance), 3), dtype=np.uint16)
        color[self.provenance == abi.GLOBAL] = (0, 0, 32768)
        m = self.provenance == abi.MEASURED
        color[m, 1] = _round_u16(65535.0 * scale[m])
        r = self.provenance == abi.REGULARIZED
        color[r, 0] = _round_u16(65535.0 * scale[r])
        color[r, 1] = _round_u16(32768.0 * scale[r])
        return encoded, color.reshape(-1)

    def visualization_samples(self) -> np.ndarray:
        """depth.rs:224-245: logarithmic depth colouring, u16[3n]."""
        log_range = np.log(self.far_depth / self.near_depth)
        has = np.isin(self.provenance, (abi.MEASURED, abi.REGULARIZED))
        out = np.zeros((len(self.provenance), 3), dtype=np.uint16)
        if has.any():
            d = self.depth[has]
            normalized = np.clip((np.log(self.far_depth) - np.log(d)) / log_range, 0.0, 1.0)
            conf = 0.45 + 0.55 * np.clip(self.confidence[has].astype(np.float32), np.float32(0),
                                         np.float32(1)).astype(np.float64)
            base = _depth_color(normalized)
            out[has] = _round_u16(base.astype(np.float64) * conf[:, None])
        out[(~has) & (self.provenance == abi.GLOBAL)] = (0, 0, 12000)
        return out.reshape(-1)

    def write_diagnostics(self, inverse_depth_path, provenance_path) -> None:
        """depth.rs:166-184: 16-bit gray inverse depth + 16-bit RGB provenance PNGs."""
        depth, prov = self.diagnostic_samples()
        _write_png16(Path(inverse_depth_path), self.columns, self.rows, depth, 1)
        _write_png16(Path(provenance_path), self.columns, self.rows, prov, 3)

    def write_visualization(self, path) -> None:
        """depth.rs:191-198."""
        _write_png16(Path(path), self.columns, self.rows, self.visualization_samples(), 3)


def _round_half_away(v):
    """Rust `round()`: half away from zero (v - trunc(v) is exact)."""
    v = np.asarray(v)
    t = np.trunc(v)
    return np.where(np.abs(v - t) >= 0.5, t + np.sign(v), t)


def _round_u16(v):
    r = _round_half_away(np.asarray(v, dtype=np.float64))
    return np.clip(np.nan_to_num(r, nan=0.0), 0, 65535).astype(np.uint16)


def _depth_color(normalized: np.ndarray) -> np.ndarray:
    """depth.rs:1861-1877."""
    stops = np.array([[0.0, 0.1, 0.7], [0.0, 0.9, 1.0], [0.0, 1.0, 0.2], [1.0, 0.9, 0.0], [1.0, 0.0, 0.0]])
    position = np.clip(normalized, 0.0, 1.0) * 4.0
    lower = np.minimum(np.floor(position).astype(np.int64), 4)
    upper = np.minimum(lower + 1, 4)
    frac = (position - lower)[:, None]
    return _round_u16((stops[lower] * (1.0 - frac) + stops[upper] * frac) * 65535.0)


def _write_png16(path: Path, width: int, height: int, samples: np.ndarray, channels: int) -> None:
    """Minimal 16-bit PNG writer (gray or RGB), written atomically."""
    data = np.asarray(samples, dtype=">u2").reshape(height, width * channels)
    raw = b"".join(b"\x00" + row.tobytes() for row in data)

    def chunk(tag: bytes, payload: bytes) -> bytes:
        return (struct.pack(">I", len(payload)) + tag + payload
                + struct.pack(">I", zlib.crc32(tag + payload) & 0xFFFFFFFF))

    color_type = 0 if channels == 1 else 2
    png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", width, height, 16, color_type, 0, 0, 0))
           + chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
    tmp = path.with_name(path.name + ".tmp")
    tmp.write_bytes(png)
    tmp.replace(path)


def output_shape(width: int, height: int, options: DepthOptions):
    """Grids of the stage: ((columns, rows, step), (coarse_columns, coarse_rows, coarse_step))
    (depth.rs:326-328 and depth.rs:726-728)."""
    coarse_step = max(options.grid_step, 4)
    step = max(coarse_step // 2, 4)
    return ((-(-width // step) + 1, -(-height // step) + 1, step),
            (-(-width // coarse_step) + 1, -(-height // coarse_step) + 1, coarse_step))


def pack_views(inputs: Sequence, alignments: Sequence):
    """Fill the C view array; returns (views, keepalive)."""
    n = len(inputs)
    views = (ViewC * n)()
    keep = []
    for i, (inp, al) in enumerate(zip(inputs, alignments)):
        luma = np.ascontiguousarray(inp.luminance.data, dtype=np.float32)
        pts = np.ascontiguousarray(al.warp.points, dtype=np.float32)
        conf = np.ascontiguousarray(al.warp.confidence, dtype=np.float32)
        keep += [luma, pts, conf]
        v = views[i]
        v.luminance = fptr(luma)
        v.luma_width = inp.luminance.width
        v.luma_height = inp.luminance.height
        v.width = inp.width
        v.height = inp.height
        v.has_camera = 1 if inp.camera is not None else 0
        v.accepted = 1 if al.report.accepted else 0
        if inp.camera is not None:
            v.camera = inp.camera.to_c()
        v.warp.step = al.warp.step
        v.warp.columns = al.warp.columns
        v.warp.rows = al.warp.rows
        v.warp.points = fptr(pts)
        v.warp.confidence = fptr(conf)
        v.warp.capacity = al.warp.columns * al.warp.rows
    return views, keep


def refine_multiview_depth(inputs: Sequence, reference_index: int, alignments: Sequence,
                           options: DepthOptions, context=None, debug=None) -> Optional[DenseDepthMap]:
    """depth.rs:312-580 on the GPU. See the module docstring for semantics.

    ``debug`` may be a dict of numpy arrays named like the fields of
    ``chiaro_depth_debug``; the library fills them with stage results.
    """
    from .runtime import default_context, pinned_pool

    if len(inputs) != len(alignments):
        return None
    if reference_index >= len(inputs) or inputs[reference_index].camera is None or not options.is_valid():
        return None
    ctx = context if context is not None else default_context()
    ref = inputs[reference_index]
    (columns, rows, step), _ = output_shape(ref.width, ref.height, options)
    m = columns * rows
    n = len(inputs)
    views, keep = pack_views(inputs, alignments)
    # outputs in page-locked host memory (a caching pool): the library copies into them at
    # the full host-link rate and overlaps the depth map's copy with the decisions
    pool = pinned_pool()
    targets = [t for t in range(n) if t != reference_index and inputs[t].camera is not None
               and alignments[t].report.accepted]
    refined = (WarpC * n)()
    out_points, out_conf = [None] * n, [None] * n
    for i in targets:
        out_points[i] = pool.empty(2 * m, np.float32)
        out_conf[i] = pool.empty(m, np.float32)
        refined[i].points = fptr(out_points[i])
        refined[i].confidence = fptr(out_conf[i])
        refined[i].capacity = m
    reports = (DepthReportC * n)()
    depth = pool.empty(m, np.float64)
    confidence = pool.empty(m, np.float32)
    provenance = pool.empty(m, np.uint8)
    dmap = DepthMapC()
    dmap.capacity = m
    dmap.depth = dptr(depth)
    dmap.confidence = fptr(confidence)
    dmap.provenance = u8ptr(provenance)
    dbg = ctx.make_debug(debug) if debug else None
    opt = options.to_c()
    status = ctx.lib.chiaro_refine_multiview_depth(ctx.handle, views, n, reference_index, C.byref(opt), refined,
                                                   reports, C.byref(dmap), C.byref(dbg) if dbg is not None else None)
    if status == abi.INVALID:
        return None
    ctx.check(status)
    for t in range(n):
        if reports[t].present:
            w = refined[t]
            alignments[t].warp = type(alignments[t].warp)(int(w.step), int(w.columns), int(w.rows),
                                                          out_points[t].reshape(m, 2), out_conf[t])
            alignments[t].report.depth = DepthAlignmentReport.from_c(reports[t])
    return DenseDepthMap(int(dmap.columns), int(dmap.rows), int(dmap.step), float(dmap.near_depth),
                         float(dmap.far_depth), depth, confidence, provenance)


class DeviceStage:
    """refine_multiview_depth (depth.rs:312-580) on device buffers, for callers that keep
    frames resident in HBM (``chiaro_refine_multiview_depth_device``).

    The luminance planes and warps of ``inputs`` / ``alignments`` are copied once into CUDA
    tensors on the context's device (``planes[i]``, ``warp_points[i]``,
    ``warp_confidence[i]``); a new frame is written into those tensors in place. Each call
    runs the stage on what they hold and writes the outputs this object owns: ``depth``
    (f64), ``confidence`` (f32) and ``provenance`` (u8) over the M output nodes, and for
    each target t (accepted, calibrated, not the reference) ``points[t]`` (f32 [M, 2]) and
    ``point_confidence[t]`` (f32 [M]); ``report(t)`` is the stage's report of target t.
    The call returns False where the reference returns None.

    ``graph=True`` enables the whole-stage CUDA graph: with unchanged views, options and
    buffers the first call launches the stage's kernels, the second captures them and
    later calls replay the graph (``graph_state``: 0, 1, 2).

    A call waits on the device for torch's current stream and returns when its outputs
    are complete.
    """

    def __init__(self, inputs: Sequence, reference_index: int, alignments: Sequence, options: DepthOptions,
                 context=None, graph: bool = False):
        import torch

        from .runtime import default_context

        if len(inputs) != len(alignments):
            raise ValueError("inputs and alignments differ in length")
        self.ctx = context if context is not None else default_context()
        self.reference_index = reference_index
        self.options = options
        device = torch.device("cuda", self.ctx.device)
        n = len(inputs)
        # the views' host pointers are replaced by device ones below, so the host copies
        # pack_views keeps alive are not needed past this point
        self.views, _ = pack_views(inputs, alignments)
        self.planes, self.warp_points, self.warp_confidence = [], [], []
        for i, (inp, al) in enumerate(zip(inputs, alignments)):
            plane = torch.from_numpy(np.ascontiguousarray(inp.luminance.data, dtype=np.float32).reshape(-1))
            points = torch.from_numpy(np.ascontiguousarray(al.warp.points, dtype=np.float32).reshape(-1))
            conf = torch.from_numpy(np.ascontiguousarray(al.warp.confidence, dtype=np.float32).reshape(-1))
            plane, points, conf = plane.to(device), points.to(device), conf.to(device)
            self.planes.append(plane)
            self.warp_points.append(points)
            self.warp_confidence.append(conf)
            self.views[i].luminance = C.cast(C.c_void_p(plane.data_ptr()), C.POINTER(C.c_float))
            self.views[i].warp.points = C.cast(C.c_void_p(points.data_ptr()), C.POINTER(C.c_float))
            self.views[i].warp.confidence = C.cast(C.c_void_p(conf.data_ptr()), C.POINTER(C.c_float))
        ref = inputs[reference_index]
        (columns, rows, _), _ = output_shape(ref.width, ref.height, options)
        self.shape = (ref.width, ref.height)
        self.nodes = m = columns * rows
        self.depth = torch.empty(m, dtype=torch.float64, device=device)
        self.confidence = torch.empty(m, dtype=torch.float32, device=device)
        self.provenance = torch.empty(m, dtype=torch.uint8, device=device)
        self.map = DepthMapC(capacity=m, depth=C.cast(C.c_void_p(self.depth.data_ptr()), C.POINTER(C.c_double)),
                             confidence=C.cast(C.c_void_p(self.confidence.data_ptr()), C.POINTER(C.c_float)),
                             provenance=C.cast(C.c_void_p(self.provenance.data_ptr()), C.POINTER(C.c_uint8)))
        self.targets = [t for t in range(n) if t != reference_index and inputs[t].camera is not None
                        and alignments[t].report.accepted]
        self.refined = (WarpC * n)()
        self.points: List = [None] * n
        self.point_confidence: List = [None] * n
        for t in self.targets:
            self.points[t] = torch.empty((m, 2), dtype=torch.float32, device=device)
            self.point_confidence[t] = torch.empty(m, dtype=torch.float32, device=device)
            self.refined[t].points = C.cast(C.c_void_p(self.points[t].data_ptr()), C.POINTER(C.c_float))
            self.refined[t].confidence = C.cast(C.c_void_p(self.point_confidence[t].data_ptr()),
                                                C.POINTER(C.c_float))
            self.refined[t].capacity = m
        self.reports = (DepthReportC * n)()
        # the library's stream, which waits for torch's current stream before each call, so
        # that plane writes queued there are seen
        self.stream = torch.cuda.ExternalStream(self.ctx.stream_handle(), device=device)
        self._device = device
        self.graph = graph

    @property
    def graph(self) -> bool:
        return self._graph

    @graph.setter
    def graph(self, enabled: bool):
        self.ctx.check(self.ctx.lib.chiaro_depth_set_stage_graph(self.ctx.handle, 1 if enabled else 0))
        self._graph = bool(enabled)

    def report(self, t: int) -> Optional[DepthAlignmentReport]:
        """The last call's report of module t (the reference's ``report.depth``), or None
        when the call did not rewrite t."""
        r = self.reports[t]
        return DepthAlignmentReport.from_c(r) if r.present else None

    @property
    def graph_state(self) -> int:
        """What the last call did: 0 launched its kernels, 1 captured the graph, 2 replayed it."""
        return int(self.ctx.lib.chiaro_depth_stage_graph_state(self.ctx.handle))

    def __call__(self, options: Optional[DepthOptions] = None) -> bool:
        """Run the stage (with ``options`` instead of the constructor's, if given; they must
        give the same output grid)."""
        options = self.options if options is None else options
        (columns, rows, _), _ = output_shape(self.shape[0], self.shape[1], options)
        if columns * rows != self.nodes:
            raise ValueError("options change the output grid")
        import torch

        self.ctx.check(self.ctx.lib.chiaro_depth_set_stage_graph(self.ctx.handle, 1 if self._graph else 0))
        self.stream.wait_stream(torch.cuda.current_stream(self._device))
        opt = options.to_c()
        status = self.ctx.lib.chiaro_refine_multiview_depth_device(
            self.ctx.handle, self.views, len(self.planes), self.reference_index, C.byref(opt), self.refined,
            self.reports, C.byref(self.map))
        if status == abi.INVALID:
            return False
        self.ctx.check(status)
        return True


class DepthPipeline:
    """refine_multiview_depth over a stream of frames of one rig, each frame's upload and the
    previous frame's read-back overlapping the current frame's stage on the GPU.

    Two ``DeviceStage`` objects on one context alternate. While frame i runs on one of them,
    frame i + 1's planes and warps go up into the other's device buffers on a copy stream, and
    frame i - 1's outputs come down from the other's output buffers into pinned host memory on
    a second copy stream. The stages themselves run one after the other (they share the
    context's working buffers), so every frame gets the bits a call of its own gives. For the
    uploads to overlap, pass pinned CPU tensors; numpy arrays are first copied into the
    pipeline's own pinned buffers on the host.
    """

    def __init__(self, inputs: Sequence, reference_index: int, alignments: Sequence, options: DepthOptions,
                 context=None):
        import torch

        from .runtime import default_context

        ctx = context if context is not None else default_context()
        self.stages = [DeviceStage(inputs, reference_index, alignments, options, context=ctx) for _ in range(2)]
        first = self.stages[0]
        self.ctx, self.targets, self.nodes = ctx, first.targets, first.nodes
        self._device = first._device
        self._in = torch.cuda.Stream(self._device)
        self._out = torch.cuda.Stream(self._device)
        self._in_ready = [torch.cuda.Event() for _ in range(2)]
        self._out_done = [torch.cuda.Event() for _ in range(2)]

        def pinned_like(t):
            return torch.empty(t.shape, dtype=t.dtype, pin_memory=True)

        # read-back buffers per stage: the host copies of its outputs
        self._host = []
        for st in self.stages:
            self._host.append({"depth": pinned_like(st.depth), "confidence": pinned_like(st.confidence),
                               "provenance": pinned_like(st.provenance),
                               "points": {t: pinned_like(st.points[t]) for t in self.targets},
                               "point_confidence": {t: pinned_like(st.point_confidence[t]) for t in self.targets}})
        # pinned staging for numpy frames, per stage: planes, warp points, warp confidence
        self._staging = [[[pinned_like(x) for x in xs] for xs in (st.planes, st.warp_points, st.warp_confidence)]
                         for st in self.stages]

    def _upload(self, k: int, frame) -> int:
        """Queue frame's host → device copies into stage k on the upload stream; returns bytes."""
        import torch

        st = self.stages[k]
        planes, points, confidence = (list(frame) + [None, None])[:3]
        moved = 0
        with torch.cuda.stream(self._in):
            for which, (srcs, dsts) in enumerate(((planes, st.planes), (points, st.warp_points),
                                                  (confidence, st.warp_confidence))):
                if srcs is None:
                    continue
                for i, (src, dst) in enumerate(zip(srcs, dsts)):
                    if not isinstance(src, torch.Tensor):
                        stage = self._staging[k][which][i]
                        stage.numpy().reshape(-1)[:] = np.asarray(src, dtype=np.float32).reshape(-1)
                        src = stage
                    dst.copy_(src.reshape(dst.shape), non_blocking=True)
                    moved += dst.numel() * dst.element_size()
            self._in_ready[k].record(self._in)
        return moved

    def _download(self, k: int) -> int:
        """Queue stage k's outputs device → pinned host on the read-back stream; returns bytes."""
        import torch

        st, host = self.stages[k], self._host[k]
        pairs = [(host["depth"], st.depth), (host["confidence"], st.confidence),
                 (host["provenance"], st.provenance)]
        pairs += [(host["points"][t], st.points[t]) for t in self.targets]
        pairs += [(host["point_confidence"][t], st.point_confidence[t]) for t in self.targets]
        with torch.cuda.stream(self._out):
            for dst, src in pairs:
                dst.copy_(src, non_blocking=True)
            self._out_done[k].record(self._out)
        return sum(src.numel() * src.element_size() for _, src in pairs)

    def _outputs(self, k: int) -> dict:
        self._out_done[k].synchronize()
        host = self._host[k]
        return {"depth": host["depth"].numpy(), "confidence": host["confidence"].numpy(),
                "provenance": host["provenance"].numpy(),
                "points": {t: v.numpy() for t, v in host["points"].items()},
                "point_confidence": {t: v.numpy() for t, v in host["point_confidence"].items()}}

    def run(self, frames: Iterable):
        """Yield (ok, outputs) per frame, in order. A frame is (planes, warp_points,
        warp_confidence), each a per-view list of host arrays or CPU tensors shaped like the
        constructor's inputs (warp_points and warp_confidence may be None: the previous warps
        stay). ok is False where the reference returns None. outputs holds numpy views of the
        pipeline's pinned read-back buffers ("depth", "confidence", "provenance", and per target
        "points" and "point_confidence"). They are reused two frames later, so copy what you
        keep. A frame's upload is queued one frame ahead and read by its own stage: leave a
        frame's host tensors unchanged until the results of the frame after it are yielded.
        ``self.bytes_up`` and ``self.bytes_down`` count the bytes each frame moved."""
        import torch

        it = iter(frames)
        current = next(it, None)
        if current is None:
            return
        self.bytes_up, self.bytes_down = [self._upload(0, current)], []
        i, pending = 0, None
        while current is not None:
            k = i % 2
            following = next(it, None)
            if following is not None:  # the other stage's last stage call has returned
                self.bytes_up.append(self._upload(1 - k, following))
            st = self.stages[k]
            st.stream.wait_event(self._in_ready[k])   # this frame's inputs are up
            st.stream.wait_event(self._out_done[k])   # frame i - 2's outputs are read back
            ok = st()
            self.bytes_down.append(self._download(k))
            if pending is not None:
                yield pending[0], self._outputs(pending[1])
            pending = (ok, k)
            current, i = following, i + 1
        yield pending[0], self._outputs(pending[1])
