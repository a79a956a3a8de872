"""Vorticity confinement (mirrors chadmv/plume src/plume/sim/vorticity.py:87-117).

The centre velocities are computed inside the curl kernel, so only the curl and the push need scratch: each
is three (nx, ny, nz) component arrays. `curl` and `push` are exposed as (nx, ny, nz, 3) views.
"""

import torch

from plume_b200 import _native as N


class VorticityConfinement:
    def __init__(self, grid):
        self._curl = torch.zeros((3, *grid.cells), dtype=torch.float32, device=grid.device)
        self._push = torch.zeros((3, *grid.cells), dtype=torch.float32, device=grid.device)

    @property
    def curl(self) -> torch.Tensor:
        return self._curl.permute(1, 2, 3, 0)

    @property
    def push(self) -> torch.Tensor:
        return self._push.permute(1, 2, 3, 0)

    def _run(self, grid, strength: float, dt: float, apply: int) -> None:
        u, v, w = (f.data for f in grid.velocity_fields())
        N.call("plume_confinement", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptrs(*self._curl), N.ptrs(*self._push),
               strength, dt, apply, N.stream())

    def apply(self, grid, strength: float, dt: float) -> None:
        """Adds strength * cell_m * (N x curl) * dt to the face velocities; nothing when strength is 0."""
        if strength == 0.0:
            return
        self._run(grid, strength, dt, 1)

    def measure_curl(self, grid) -> torch.Tensor:
        """The curl of the grid's current velocity at cell centres."""
        self._run(grid, 0.0, 0.0, 0)
        return self.curl
