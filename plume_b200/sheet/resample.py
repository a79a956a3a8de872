"""Tap tables of the bicubic resampling the reference's sheet uses (chadmv/plume src/plume/sheet/resample.py:16-41,
which calls Pillow's Image.resize(BICUBIC, box) on float32 images).

This is Pillow's published separable algorithm: for each output index, the window of source indices within the
filter's support (2, widened by the scale when shrinking) around the output's centre in the source, with
bicubic weights (a = -0.5) normalised to sum to 1. Pillow takes the box as float32, so the box edges and their
difference are float32 and the rest is double. The device kernels apply the tables (sheet.cu).
"""

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Taps:
    first: np.ndarray    # int32 (out,): first source index
    count: np.ndarray    # int32 (out,): window length
    weights: np.ndarray  # float64 (out, ksize)

    @property
    def ksize(self) -> int:
        return self.weights.shape[1]


def _bicubic(x: np.ndarray) -> np.ndarray:
    a = -0.5
    x = np.abs(x)
    inner = ((a + 2.0) * x - (a + 3.0)) * x * x + 1
    outer = (((x - 5) * x + 8) * x - 4) * a
    return np.where(x < 1.0, inner, np.where(x < 2.0, outer, 0.0))


def taps(in_size: int, in0: float, in1: float, out_size: int) -> Taps:
    f0, f1 = np.float32(in0), np.float32(in1)
    scale = filterscale = float(np.float32(f1 - f0)) / out_size
    if filterscale < 1.0:
        filterscale = 1.0
    support = 2.0 * filterscale
    ksize = int(math.ceil(support)) * 2 + 1
    center = float(f0) + (np.arange(out_size, dtype=np.float64) + 0.5) * scale
    ss = 1.0 / filterscale
    first = np.maximum(np.trunc(center - support + 0.5).astype(np.int64), 0)
    last = np.minimum(np.trunc(center + support + 0.5).astype(np.int64), in_size)
    count = np.maximum(last - first, 0)
    weights = np.zeros((out_size, ksize), dtype=np.float64)
    total = np.zeros(out_size, dtype=np.float64)
    for x in range(ksize):
        live = x < count
        w = np.where(live, _bicubic((x + first - center + 0.5) * ss), 0.0)
        weights[:, x] = w
        total = total + w
    safe = np.where(total != 0.0, total, 1.0)
    weights = np.where((np.arange(ksize)[None, :] < count[:, None]) & (total[:, None] != 0.0),
                       weights / safe[:, None], weights)
    return Taps(first.astype(np.int32), count.astype(np.int32), weights)


def identity(size: int) -> Taps:
    """The table of a pass Pillow skips (each output copies its own source index)."""
    return Taps(np.arange(size, dtype=np.int32), np.ones(size, dtype=np.int32), np.ones((size, 1), dtype=np.float64))
