"""The blurred-smoke gradient used for the normal layout (mirrors chadmv/plume
src/plume/render/normal_field.py:41-69): three separable Gaussian passes (radius ceil(3 sigma), edge clamp)
then per-cell central differences. `gradient` is (nx, ny, nz, 3)."""

import math

import ctypes

import numpy as np
import torch

from plume_b200 import _native as N


class NormalField:
    def __init__(self, cells, blur_cells: float, device: str):
        self.device = device
        self.blurred = torch.zeros(tuple(cells), dtype=torch.float32, device=device)
        self.scratch = torch.zeros(tuple(cells), dtype=torch.float32, device=device)
        self.gradient = torch.zeros((*cells, 3), dtype=torch.float32, device=device)
        self.radius = math.ceil(3.0 * blur_cells) if blur_cells > 0 else 0
        self.weights = _gaussian_weights(blur_cells, self.radius)

    def compute(self, smoke: torch.Tensor) -> torch.Tensor:
        weights = (ctypes.c_float * len(self.weights))(*self.weights.tolist())
        N.call("plume_normal_field", N.shape3(smoke), N.field_ptr(smoke), N.storage_of(smoke), N.ptr(self.blurred),
               N.ptr(self.scratch),
               N.ptr(self.gradient), weights, self.radius, N.stream())
        return self.gradient


def _gaussian_weights(sigma: float, radius: int) -> np.ndarray:
    if radius == 0:
        return np.ones(1, dtype=np.float32)
    offsets = np.arange(-radius, radius + 1, dtype=np.float64)
    weights = np.exp(-offsets**2 / (2.0 * sigma**2))
    return (weights / weights.sum()).astype(np.float32)
