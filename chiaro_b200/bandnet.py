"""The learned band proposal of the banded SGM (no counterpart in the reference).

A small convolutional network (six 3x3 convolutions of 32 channels on the coarse
grid, bf16 tensor-core kernels with fp32 accumulation, ``chiaro_bandnet_*`` in the
library) predicts each node's label from the reference luminance and a 16-bin
summary of its costs. Per tile, the band of ``band`` labels is centred on the
tile's mean prediction, and ``chiaro_sgm_banded`` aggregates only those labels,
falling back to a windowed full-range SGM where the winner sits on a band edge.
Training targets are the exact full-range SGM's winners (``samples_from_stage``).
Device memory is torch's; the computation is the library's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

LAYERS, CH, TAPS = 6, 32, 9


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised fp32 parameters in the library's layout (per layer [tap][co][ci] then 32 biases).
    The first layer sees 17 live input channels; the last layer's channel 0 starts near the label range's middle."""
    rng = np.random.default_rng(seed)
    parts = []
    for layer in range(LAYERS):
        fan_in = TAPS * (17 if layer == 0 else CH)
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), (TAPS, CH, CH)).astype(np.float32)
        if layer == 0:
            w[:, :, 17:] = 0.0
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

    costs: np.ndarray      # [N * D] f32
    guidance: np.ndarray   # [N] f32
    winners: np.ndarray    # [N] int32
    mask: np.ndarray       # [N] uint8
    columns: int
    rows: int
    labels: int


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
        assert all((s.columns, s.rows, s.labels) == (first.columns, first.rows, first.labels) for s in samples)
        costs = t.from_numpy(np.concatenate([s.costs for s in samples])).to(self.device)
        guidance = t.from_numpy(np.concatenate([s.guidance for s in samples])).to(self.device)
        winners = t.from_numpy(np.concatenate([s.winners for s in samples])).to(self.device)
        mask = t.from_numpy(np.concatenate([s.mask for s in samples])).to(self.device)
        return costs, guidance, winners, mask, first

    def train(self, samples: List[Sample], steps: int, learning_rate: float = 2e-3) -> np.ndarray:
        costs, guidance, winners, mask, s = self._batch(samples)
        losses = np.zeros(steps, np.float32)
        self.ctx.check(self.ctx.lib.chiaro_bandnet_train_device(
            self.ctx.handle, self.params.data_ptr(), self.m.data_ptr(), self.v.data_ptr(), self.step, steps,
            costs.data_ptr(), guidance.data_ptr(), winners.data_ptr(), mask.data_ptr(), len(samples), s.columns,
            s.rows, s.labels, learning_rate, losses.ctypes.data_as(C.POINTER(C.c_float))))
        self.step += steps
        return losses

    def gradient(self, samples: List[Sample]):
        costs, guidance, winners, mask, s = self._batch(samples)
        grads = self.torch.empty_like(self.params)
        loss = C.c_float()
        self.ctx.check(self.ctx.lib.chiaro_bandnet_gradient_device(
            self.ctx.handle, self.params.data_ptr(), costs.data_ptr(), guidance.data_ptr(), winners.data_ptr(),
            mask.data_ptr(), len(samples), s.columns, s.rows, s.labels, grads.data_ptr(), C.byref(loss)))
        return grads.cpu().numpy(), float(loss.value)

    def propose(self, costs, guidance, columns: int, rows: int, labels: int, tile: int = 4, band: int = 24,
                centres: Optional[object] = None):
        """Tile offsets (a device int32 tensor) for chiaro_sgm_banded_device; costs and guidance are
        device tensors of one image."""
        t = self.torch
        tiles = (-(-columns // tile)) * (-(-rows // tile))
        offsets = t.empty(tiles, dtype=t.int32, device=self.device)
        self.ctx.check(self.ctx.lib.chiaro_bandnet_propose_device(
            self.ctx.handle, self.params.data_ptr(), costs.data_ptr(), guidance.data_ptr(), columns, rows, labels,
            tile, band, offsets.data_ptr(), centres.data_ptr() if centres is not None else None))
        return offsets
