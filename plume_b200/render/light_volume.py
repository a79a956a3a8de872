"""The light volume (mirrors chadmv/plume src/plume/render/light_volume.py:36-51): the share of the key light
reaching each cell through the smoke toward the light, exp(-opacity_per_density * column density)."""

import numpy as np
import torch

from plume_b200 import _native as N


class LightVolume:
    def __init__(self, cells, toward_light_world, opacity_per_density: float, device: str):
        self.device = device
        direction = np.asarray(toward_light_world, dtype=np.float64)
        self.toward_light = tuple(float(x) for x in direction / np.linalg.norm(direction))
        self.opacity_per_density = opacity_per_density
        self.light = torch.zeros(tuple(cells), dtype=torch.float32, device=device)
        # per-frame map of each 4x4x4 brick's largest smoke value: the march skips samples that add nothing
        self.bricks = torch.empty(N.lib().plume_brick_floats(N.c_int3(*cells)), dtype=torch.float32, device=device)

    def compute(self, smoke: torch.Tensor, cell_m: float, march_cells: bool = False) -> torch.Tensor:
        """The light volume of `smoke`. With `march_cells`, only the cells a camera march of this same smoke
        reads get their value (bit for bit) and the rest hold 1: what FrameRenderer.prepare needs."""
        N.call("plume_march_light_volume" if march_cells else "plume_light_volume", N.shape3(smoke),
               N.field_ptr(smoke), N.storage_of(smoke), N.f3(self.toward_light), cell_m,
               self.opacity_per_density, N.ptr(self.light), N.ptr(self.bricks), N.stream())
        return self.light
