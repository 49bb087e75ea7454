"""The learned band proposal of the banded SGM (no counterpart in the reference).

A small convolutional network (six 3x3 convolutions of 32 channels on the coarse
grid, bf16 tensor-core kernels with fp32 accumulation, ``chiaro_bandnet_*`` in the
library) predicts each node's label from the reference luminance and the costs of
16 sampled labels (the coarse search's pre-pass, ``coarse.band_prepass``). Per
tile, the band of ``band`` labels is centred on the tile's mean prediction; the
learned-band coarse search (``coarse.coarse_depth``) scores and aggregates only
those labels, searching the full range again where a tile's winner sits on a band
edge or fails the cross-view check. Training targets are the exact full-range
search's winners (``samples_from_prepass`` or ``samples_from_stage``). Device
memory is torch's; the computation is the library's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import band as bandmod

LAYERS, CH, TAPS = 6, 32, 9
INPUTS = 19  # live input channels: guidance, 16 cost bins, the cost argmin and the minimum cost


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised fp32 parameters in the library's layout (per layer [tap][co][ci] then 32 biases).
    The first layer sees INPUTS live input channels; the last layer's channel 0 starts near the label range's middle."""
    rng = np.random.default_rng(seed)
    parts = []
    for layer in range(LAYERS):
        fan_in = TAPS * (INPUTS if layer == 0 else CH)
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), (TAPS, CH, CH)).astype(np.float32)
        if layer == 0:
            w[:, :, INPUTS:] = 0.0
        b = np.zeros(CH, np.float32)
        if layer == LAYERS - 1:
            w *= 0.1
            b[0] = 0.5
        parts += [w.reshape(-1), b]
    return np.concatenate(parts)


@dataclass
class Sample:
    """One training or evaluation image: the coarse grid's cost volume, guidance,
    the full-range SGM's winners and the mask of scored (tested) nodes."""

    costs: np.ndarray      # [N * stride] f32: full rows (stride D) or the pre-pass's rows (stride 17)
    guidance: np.ndarray   # [N] f32
    winners: np.ndarray    # [N] int32
    mask: np.ndarray       # [N] uint8
    columns: int
    rows: int
    labels: int
    stride: int = 0        # 0: full rows (labels)

    @property
    def cost_stride(self) -> int:
        return self.stride or self.labels


def samples_from_stage(scene, context=None) -> Sample:
    """Run the exact GPU stage on a scene and keep its coarse cost volume and SGM winners."""
    from .depth import output_shape, refine_multiview_depth
    (_, _, _), (cc, cr, _) = output_shape(scene.width, scene.height, scene.options)
    n, d = cc * cr, scene.options.planes + 1
    dbg = {"coarse_costs": np.zeros(n * d, np.float32), "coarse_guidance": np.zeros(n, np.float32),
           "regularised": np.zeros(n * d, np.float32), "coarse_tested": np.zeros(n, np.uint8)}
    refine_multiview_depth(scene.inputs(), scene.reference_index, scene.alignments(), scene.options,
                           context=context, debug=dbg)
    winners = (1 + np.argmin(dbg["regularised"].reshape(n, d)[:, 1:], axis=1)).astype(np.int32)
    return Sample(dbg["coarse_costs"], dbg["coarse_guidance"], winners, dbg["coarse_tested"], cc, cr, d)


def samples_from_prepass(stage, options=None) -> Sample:
    """One training image from a DeviceStage's views, all on the GPU: the pre-pass's rows
    (the network's inputs at inference) and the exact plain coarse search's winners."""
    from .coarse import PREPASS_SLOTS, band_prepass, coarse_depth
    options = options or stage.options
    costs, guidance, _ = band_prepass(stage, options)
    plain = coarse_depth(stage, None, options)
    return Sample(costs.cpu().numpy().reshape(-1), guidance.cpu().numpy(), plain.winner.cpu().numpy(),
                  plain.tested.cpu().numpy(), plain.columns, plain.rows, plain.labels, PREPASS_SLOTS)


def tile_targets(sample: Sample, tile: int = 4, kind: str = "median") -> Sample:
    """The band network's training targets: every node of a tile learns one label of the
    tile's tested winners, their median (``kind="median"``: the band holds the tile's main
    surface) or the middle of their range (``"midrange"``: a band centred there covers the
    tile whenever the range fits in it); a tile with no tested node learns label 1, where
    flat costs need no fallback."""
    if kind not in ("median", "midrange"):
        raise ValueError(f"unknown target kind {kind!r}")
    columns, rows = sample.columns, sample.rows
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    winners = sample.winners.reshape(rows, columns)
    tested = sample.mask.reshape(rows, columns).astype(bool)
    out = np.ones((rows, columns), np.int32)
    for y in range(ty):
        for x in range(tx):
            block = (slice(y * tile, (y + 1) * tile), slice(x * tile, (x + 1) * tile))
            w = winners[block][tested[block]]
            if w.size:
                out[block] = int(np.rint(np.median(w))) if kind == "median" else (int(w.min()) + int(w.max())) // 2
    return Sample(sample.costs, sample.guidance, out.reshape(-1), np.ones(columns * rows, np.uint8), columns, rows,
                  sample.labels, sample.stride)


def wide_tile_fraction(sample: Sample, tile: int = 4, band: int = 24) -> float:
    """The share of tiles whose tested full-range winners span more than band - 3 labels:
    no band of ``band`` labels holds all of them off its edges, so every proposal method
    falls back there or disagrees with the full-range SGM."""
    tx, ty = bandmod.tiles_of(sample.columns, sample.rows, tile)
    winners = sample.winners.reshape(sample.rows, sample.columns)
    tested = sample.mask.reshape(sample.rows, sample.columns).astype(bool)
    wide = 0
    for y in range(ty):
        for x in range(tx):
            block = (slice(y * tile, (y + 1) * tile), slice(x * tile, (x + 1) * tile))
            w = winners[block][tested[block]]
            wide += int(w.size > 0 and int(w.max()) - int(w.min()) > band - 3)
    return wide / (tx * ty)


class BandNet:
    """Parameters and Adam state on the device; training and proposals through the library."""

    def __init__(self, context, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.ctx = context
        self.device = torch.device("cuda", device)
        count = int(context.lib.chiaro_bandnet_parameter_count())
        params = init_params(seed)
        assert params.size == count
        self.params = torch.from_numpy(params).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0

    def _batch(self, samples: List[Sample]):
        t = self.torch
        first = samples[0]
        assert all((s.columns, s.rows, s.labels, s.cost_stride) == (first.columns, first.rows, first.labels,
                                                                   first.cost_stride) for s in samples)
        def cat(arrays):  # numpy arrays, or device tensors kept on the device
            if isinstance(arrays[0], np.ndarray):
                return t.from_numpy(np.concatenate(arrays)).to(self.device)
            return t.cat([a.reshape(-1) for a in arrays]).to(self.device)

        costs = cat([s.costs for s in samples])
        guidance = cat([s.guidance for s in samples])
        winners = cat([s.winners for s in samples])
        mask = cat([s.mask for s in samples])
        return costs, guidance, winners, mask, first

    # ---- checkpoint: a versioned binary of the parameters and the optimiser state --------
    MAGIC = b"CHBN"
    VERSION = 1

    def save(self, path, meta: Optional[dict] = None) -> None:
        """Write the parameters, Adam moments and step to ``path`` (binary: magic, version,
        count, step, then three float32 arrays) and ``meta`` to ``path`` + ".json"."""
        import json
        import struct
        from pathlib import Path as _Path
        path = _Path(path)
        arrays = [x.detach().cpu().numpy().astype(np.float32) for x in (self.params, self.m, self.v)]
        with open(path, "wb") as f:
            f.write(self.MAGIC + struct.pack("<IQQ", self.VERSION, arrays[0].size, self.step))
            for a in arrays:
                f.write(a.tobytes())
        info = dict(meta or {})
        info.update({"format": "CHBN", "version": self.VERSION, "parameters": int(arrays[0].size),
                     "step": int(self.step), "layers": LAYERS, "channels": CH, "inputs": INPUTS})
        path.with_suffix(path.suffix + ".json").write_text(json.dumps(info, indent=1) + "\n")

    def load(self, path) -> dict:
        """Read a checkpoint written by ``save`` (resuming its optimiser state); returns its metadata."""
        import json
        import struct
        from pathlib import Path as _Path
        path = _Path(path)
        data = path.read_bytes()
        if data[:4] != self.MAGIC:
            raise ValueError(f"{path}: not a band network checkpoint")
        version, count, step = struct.unpack("<IQQ", data[4:24])
        if version != self.VERSION or count != self.params.numel():
            raise ValueError(f"{path}: version {version} with {count} parameters, expected version "
                             f"{self.VERSION} with {self.params.numel()}")
        arrays = np.frombuffer(data[24:24 + 12 * count], np.float32).reshape(3, count)
        for dst, src in zip((self.params, self.m, self.v), arrays):
            dst.copy_(self.torch.from_numpy(src.copy()))
        self.step = int(step)
        meta = path.with_suffix(path.suffix + ".json")
        return json.loads(meta.read_text()) if meta.exists() else {}

    def train(self, samples: List[Sample], steps: int, learning_rate: float = 2e-3) -> np.ndarray:
        costs, guidance, winners, mask, s = self._batch(samples)
        losses = np.zeros(steps, np.float32)
        self.ctx.check(self.ctx.lib.chiaro_bandnet_train_device(
            self.ctx.handle, self.params.data_ptr(), self.m.data_ptr(), self.v.data_ptr(), self.step, steps,
            costs.data_ptr(), guidance.data_ptr(), winners.data_ptr(), mask.data_ptr(), len(samples), s.columns,
            s.rows, s.labels, s.cost_stride, learning_rate, losses.ctypes.data_as(C.POINTER(C.c_float))))
        self.step += steps
        return losses

    def gradient(self, samples: List[Sample]):
        costs, guidance, winners, mask, s = self._batch(samples)
        grads = self.torch.empty_like(self.params)
        loss = C.c_float()
        self.ctx.check(self.ctx.lib.chiaro_bandnet_gradient_device(
            self.ctx.handle, self.params.data_ptr(), costs.data_ptr(), guidance.data_ptr(), winners.data_ptr(),
            mask.data_ptr(), len(samples), s.columns, s.rows, s.labels, s.cost_stride, grads.data_ptr(),
            C.byref(loss)))
        return grads.cpu().numpy(), float(loss.value)

    def propose(self, costs, guidance, columns: int, rows: int, labels: int, tile: int = 4, band: int = 24,
                centres: Optional[object] = None, stride: int = 0):
        """Tile offsets (a device int32 tensor) for chiaro_sgm_banded_device; costs (full rows, or
        the pre-pass's with stride 17) and guidance are device tensors of one image."""
        t = self.torch
        tiles = (-(-columns // tile)) * (-(-rows // tile))
        offsets = t.empty(tiles, dtype=t.int32, device=self.device)
        self.ctx.check(self.ctx.lib.chiaro_bandnet_propose_device(
            self.ctx.handle, self.params.data_ptr(), costs.data_ptr(), guidance.data_ptr(), columns, rows, labels,
            stride or labels, tile, band, offsets.data_ptr(), centres.data_ptr() if centres is not None else None))
        return offsets


def _render(name: str, seed: int, overrides: dict):
    from . import scenes
    return scenes.workload(name, seed=seed, cache=False, **overrides)


def render_scenes(name: str, seeds, processes: Optional[int] = None, **overrides):
    """Render seeded workloads in spawned worker processes (the renderer is numpy on the host;
    spawned workers are safe after CUDA is initialised in this process). Where workers cannot
    start (a caller whose main module cannot be re-imported), the scenes render here in turn."""
    import multiprocessing as mp
    import os
    from concurrent.futures import ProcessPoolExecutor
    from concurrent.futures.process import BrokenProcessPool
    seeds = list(seeds)
    processes = processes or max(1, min(len(seeds), os.cpu_count() or 1, 16))
    if processes > 1:
        try:
            with ProcessPoolExecutor(processes, mp_context=mp.get_context("spawn")) as pool:
                return list(pool.map(_render, [name] * len(seeds), seeds, [overrides] * len(seeds)))
        except BrokenProcessPool:
            pass
    return [_render(name, s, overrides) for s in seeds]


def band_winners(context, costs, guidance, columns: int, rows: int, labels: int, offsets, tile: int = 4,
                 band: int = 24, margin: int = 16):
    """chiaro_sgm_banded_device on device tensors: (winner labels, fallback flags per tile) as numpy."""
    import torch
    tx, ty = bandmod.tiles_of(columns, rows, tile)
    if isinstance(offsets, np.ndarray):
        offsets = torch.from_numpy(np.ascontiguousarray(offsets, np.int32)).to(costs.device)
    winner = torch.empty(columns * rows, dtype=torch.int32, device=costs.device)
    fallback = torch.empty(tx * ty, dtype=torch.uint8, device=costs.device)
    context.check(context.lib.chiaro_sgm_banded_device(
        context.handle, costs.data_ptr(), guidance.data_ptr(), columns, rows, labels, offsets.data_ptr(), tile, band,
        margin, winner.data_ptr(), fallback.data_ptr()))
    return winner.cpu().numpy(), fallback.cpu().numpy()


@dataclass
class BandScore:
    """Winner agreement of a banded SGM with the full-range SGM, summed over images."""

    nodes: int = 0
    exact: int = 0
    within_one: int = 0
    tested: int = 0
    tested_exact: int = 0
    tested_within_one: int = 0
    tiles: int = 0
    fallback_tiles: int = 0
    windows: int = 0

    def add(self, winners: np.ndarray, fallback: np.ndarray, sample: Sample) -> None:
        diff = np.abs(winners.astype(np.int64) - sample.winners)
        tested = sample.mask.astype(bool)
        self.nodes += diff.size
        self.exact += int((diff == 0).sum())
        self.within_one += int((diff <= 1).sum())
        self.tested += int(tested.sum())
        self.tested_exact += int((diff[tested] == 0).sum())
        self.tested_within_one += int((diff[tested] <= 1).sum())
        self.tiles += fallback.size
        self.fallback_tiles += int(fallback.sum())

    def summary(self) -> dict:
        rate = lambda a, b: round(a / b, 5) if b else None
        return {"within_one_plane": rate(self.tested_within_one, self.tested),
                "exact": rate(self.tested_exact, self.tested),
                "within_one_plane_all_nodes": rate(self.within_one, self.nodes),
                "fallback_rate": rate(self.fallback_tiles, self.tiles),
                "fallback_windows": self.windows, "tested_nodes": self.tested, "tiles": self.tiles}


def evaluate(context, samples: List[Sample], nets: Optional[dict] = None, tile: int = 4, band: int = 24,
             margin: int = 16) -> dict:
    """Banded SGM with fallback against the full-range SGM's winners on each sample: with the
    naive bands (the median cost argmin of each tile) and with each network of ``nets``
    ({name: BandNet}). Agreement is over the tested nodes (those with a finite cost)."""
    import torch
    nets = nets or {}
    device = torch.device("cuda", 0) if not nets else next(iter(nets.values())).device
    scores = {"naive": BandScore(), **{name: BandScore() for name in nets}}
    for s in samples:
        costs = torch.from_numpy(s.costs).to(device)
        guidance = torch.from_numpy(s.guidance).to(device)
        proposals = {"naive": bandmod.naive_tile_offsets(s.costs, s.columns, s.rows, s.labels, tile, band)}
        for name, net in nets.items():
            proposals[name] = net.propose(costs, guidance, s.columns, s.rows, s.labels, tile, band)
        for kind, offsets in proposals.items():
            w, f = band_winners(context, costs, guidance, s.columns, s.rows, s.labels, offsets, tile, band, margin)
            scores[kind].add(w, f, s)
            windows = C.c_int()
            context.check(context.lib.chiaro_sgm_banded_report(context.handle, C.byref(windows)))
            scores[kind].windows += windows.value
    return {k: v.summary() for k, v in scores.items()}


def evaluate_search(stages, nets: Optional[dict] = None, tile: int = 4, band: int = 24, margin: int = 8,
                    fraction: float = 0.5) -> dict:
    """The learned-band coarse search against the plain search on each DeviceStage: the
    naive band and each network of ``nets`` ({name: BandNet}), scored by the agreement of
    their winners with the plain search's within one plane over the tested nodes, the
    fallback rate (tiles searched again at full range; edge and cross-view counts) and
    the search times, summed over the stages."""
    from .coarse import BandOptions, coarse_depth
    nets = nets or {}
    kinds = {"naive": None, **{name: net.params for name, net in nets.items()}}
    totals = {k: dict(tested=0, exact=0, within_one=0, tiles=0, fallback=0, edge=0, consistency=0, windows=0,
                      window_nodes=0, ms=0.0, ms_phases={}) for k in kinds}
    plain_ms, plain_phases = 0.0, {}
    for stage in stages:
        plain = coarse_depth(stage)
        winners = plain.winner.cpu().numpy().astype(np.int64)
        tested = plain.tested.cpu().numpy().astype(bool)
        plain_ms += plain.report["ms"]["total"]
        for k, v in plain.report["ms"].items():
            plain_phases[k] = plain_phases.get(k, 0.0) + v
        for kind, params in kinds.items():
            r = coarse_depth(stage, BandOptions(params, tile, band, margin, fraction))
            diff = np.abs(r.winner.cpu().numpy().astype(np.int64) - winners)[tested]
            t = totals[kind]
            t["tested"] += int(tested.sum())
            t["exact"] += int((diff == 0).sum())
            t["within_one"] += int((diff <= 1).sum())
            rep = r.report
            t["tiles"] += rep["tiles"]
            t["fallback"] += rep["fallback_tiles"]
            t["edge"] += rep["edge_tiles"]
            t["consistency"] += rep["consistency_tiles"]
            t["windows"] += rep["windows"]
            t["window_nodes"] += rep["window_nodes"]
            t["ms"] += rep["ms"]["total"]
            for k, v in rep["ms"].items():
                t["ms_phases"][k] = t["ms_phases"].get(k, 0.0) + v
    rate = lambda a, b: round(a / b, 5) if b else None
    out = {"plain_ms": round(plain_ms, 3), "plain_ms_phases": {k: round(v, 3) for k, v in plain_phases.items()}}
    for kind, t in totals.items():
        out[kind] = {"within_one_plane": rate(t["within_one"], t["tested"]), "exact": rate(t["exact"], t["tested"]),
                     "fallback_rate": rate(t["fallback"], t["tiles"]), "edge_rate": rate(t["edge"], t["tiles"]),
                     "consistency_rate": rate(t["consistency"], t["tiles"]), "windows": t["windows"],
                     "window_nodes": t["window_nodes"], "ms": round(t["ms"], 3),
                     "speedup_vs_plain": round(plain_ms / t["ms"], 3) if t["ms"] else None,
                     "ms_phases": {k: round(v, 3) for k, v in t["ms_phases"].items()}}
    return out
