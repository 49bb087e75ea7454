"""Image containers on the host: ``Plane`` (crates/chiaro-fusion/src/image.rs:431-514).

``Plane.sample`` is the bilinear texel fetch of image.rs:451-466, written with
numpy float32 scalars so it rounds as the Rust code does. The depth kernels
carry their own device copy of it.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

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
