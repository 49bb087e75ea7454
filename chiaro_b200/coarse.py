"""The coarse depth search as an operator: plain, or with the learned band.

``coarse_depth(stage)`` runs the stage's coarse search (build_cost_volume,
semi_global_costs and each coarse node's winning label; crates/chiaro-fusion/src/
depth.rs:1187-1413) on a ``DeviceStage``'s device-resident views, through
``chiaro_coarse_depth_device``. With ``band=BandOptions(...)`` it runs the
learned-band form instead (no counterpart in the reference): a pre-pass of 16
sampled labels, a band per tile from the band network (or, without parameters, the
tile's median sampled winner), the banded cost volume and SGM, and a full-range
search in windows around the tiles whose winner sits on a band edge or that fail
the cross-view check. ``band_prepass(stage)`` returns the pre-pass alone: the
network's inputs, for training it. Device memory is torch's; the computation is
the library's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

from . import abi
from .band import tiles_of
from .depth import DepthOptions, output_shape

PREPASS_SLOTS = 17  # label 0 and the 16 sampled labels


def sample_labels(labels: int):
    """The pre-pass's 16 sampled labels of a D-label volume (first and last finite label included)."""
    return [1 + (b * (labels - 2) + 7) // 15 for b in range(16)]


@dataclass
class BandOptions:
    """chiaro_band_options. ``params``: a device tensor of the network's parameters, or None
    for the naive band."""

    params: Optional[object] = None
    tile: int = 4
    band: int = 24
    margin: int = 8
    contradicted_fraction: float = 0.5

    def to_c(self) -> abi.BandOptionsC:
        return abi.BandOptionsC(self.params.data_ptr() if self.params is not None else None, self.tile, self.band,
                                self.margin, float(self.contradicted_fraction), 0)


@dataclass
class CoarseResult:
    """Winners ([N] int32, device), tested flags ([N] uint8, device), and for the banded
    form each tile's band start and fallback flag ([tiles], device) and the report."""

    columns: int
    rows: int
    labels: int
    winner: object
    tested: object
    offsets: Optional[object] = None
    fallback: Optional[object] = None
    report: Optional[dict] = None


def _grid(stage, options: DepthOptions):
    _, (columns, rows, _) = output_shape(stage.shape[0], stage.shape[1], options)
    return columns, rows, options.planes + 1


def coarse_depth(stage, band: Optional[BandOptions] = None, options: Optional[DepthOptions] = None) -> CoarseResult:
    """chiaro_coarse_depth_device on a DeviceStage's views (their current contents)."""
    import torch
    options = options or stage.options
    ctx = stage.ctx
    columns, rows, labels = _grid(stage, options)
    n = columns * rows
    device = stage._device
    winner = torch.empty(n, dtype=torch.int32, device=device)
    tested = torch.empty(n, dtype=torch.uint8, device=device)
    offsets = fallback = None
    report = abi.BandReportC()
    band_c = None
    if band is not None:
        tx, ty = tiles_of(columns, rows, max(int(band.tile), 1))  # a bad tile is the library's to refuse
        offsets = torch.empty(tx * ty, dtype=torch.int32, device=device)
        fallback = torch.empty(tx * ty, dtype=torch.uint8, device=device)
        band_c = band.to_c()
    stage.stream.wait_stream(torch.cuda.current_stream(device))
    opt = options.to_c()
    status = ctx.lib.chiaro_coarse_depth_device(
        ctx.handle, stage.views, len(stage.planes), stage.reference_index, C.byref(opt),
        C.byref(band_c) if band_c is not None else None, winner.data_ptr(), tested.data_ptr(),
        offsets.data_ptr() if offsets is not None else None, fallback.data_ptr() if fallback is not None else None,
        C.byref(report))
    ctx.check(status)
    names = ("setup", "prepass", "proposal", "cost_volume", "sgm", "fallback", "total")
    rep = {"tiles": report.tiles, "edge_tiles": report.edge_tiles, "consistency_tiles": report.consistency_tiles,
           "fallback_tiles": report.fallback_tiles, "windows": report.windows, "window_nodes": report.window_nodes,
           "ms": {k: float(report.ms[i]) for i, k in enumerate(names)}}
    return CoarseResult(columns, rows, labels, winner, tested, offsets, fallback, rep)


def band_prepass(stage, options: Optional[DepthOptions] = None):
    """The pre-pass alone: (sampled costs [N, 17], guidance [N], tested [N]) device tensors."""
    import torch
    options = options or stage.options
    ctx = stage.ctx
    columns, rows, _ = _grid(stage, options)
    n = columns * rows
    device = stage._device
    costs = torch.empty((n, PREPASS_SLOTS), dtype=torch.float32, device=device)
    guidance = torch.empty(n, dtype=torch.float32, device=device)
    tested = torch.empty(n, dtype=torch.uint8, device=device)
    stage.stream.wait_stream(torch.cuda.current_stream(device))
    opt = options.to_c()
    ctx.check(ctx.lib.chiaro_band_prepass_device(ctx.handle, stage.views, len(stage.planes), stage.reference_index,
                                                 C.byref(opt), costs.data_ptr(), guidance.data_ptr(),
                                                 tested.data_ptr()))
    return costs, guidance, tested
