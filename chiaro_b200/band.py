"""Band proposals for the banded SGM (chiaro_sgm_banded): per tile of tile x tile
coarse nodes, the offset O of the label window [O, O + band).

``naive_tile_offsets`` is the baseline without learning: the median over the
tile of each node's cost argmin (labels 1..D-1), centred in the band.
"""
from __future__ import annotations

import numpy as np


def tiles_of(columns: int, rows: int, tile: int):
    return -(-columns // tile), -(-rows // tile)


def centred_offsets(centres: np.ndarray, labels: int, band: int) -> np.ndarray:
    """Offsets that centre the band on per-tile label centres, clamped to [1, D - band]."""
    return np.clip(np.rint(centres).astype(np.int64) - band // 2, 1, labels - band).astype(np.int32)


def naive_tile_offsets(costs: np.ndarray, columns: int, rows: int, labels: int, tile: int = 4,
                       band: int = 24) -> np.ndarray:
    argmin = 1 + np.argmin(np.asarray(costs, np.float32).reshape(rows, columns, labels)[:, :, 1:], axis=2)
    tx, ty = tiles_of(columns, rows, tile)
    centres = np.empty(ty * tx)
    for y in range(ty):
        for x in range(tx):
            centres[y * tx + x] = np.median(argmin[y * tile:(y + 1) * tile, x * tile:(x + 1) * tile])
    return centred_offsets(centres, labels, band)
