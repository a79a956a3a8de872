"""The CFL cap (mirrors chadmv/plume src/plume/sim/step_cap.py:22-66).

Before each block of steps the cap measures the fastest face velocity component and the fastest active
emitter and splits the block so the fastest gas crosses at most `max_cells_per_step` cells per step. The
grid's fastest speed is a device max-reduction (exact in any order); only its 4 bytes come back.
"""

import math
from dataclasses import dataclass

import numpy as np
import torch

from plume_b200 import _native as N
from plume_b200.recipe.errors import RecipeError


@dataclass(frozen=True)
class StepPlan:
    steps: int
    speed_mps: float


class StepCap:
    def __init__(self, recipe):
        self.cell_m = recipe.domain.cell_m
        self.max_cells = recipe.solver.max_cells_per_step
        self.max_substeps = recipe.solver.max_substeps
        self.emitters = [(e.start_s, e.end_s, _emitter_speed(e.velocity_mps, e.velocity_mode))
                         for e in recipe.emitter]

    def plan(self, grid, start_s: float, length_s: float, base_steps: int, label: str) -> StepPlan:
        return self.plan_for_speed(self.grid_speed(grid), start_s, length_s, base_steps, label)

    def plan_for_speed(self, grid_speed: float, start_s: float, length_s: float, base_steps: int,
                       label: str) -> StepPlan:
        """The plan for a block given the grid's fastest face speed (read by the caller, e.g. for many grids
        at once)."""
        speed = max(grid_speed, self.emitter_speed(start_s, start_s + length_s))
        needed = math.ceil(speed * length_s / (self.max_cells * self.cell_m))
        steps = max(base_steps, needed)
        if steps > max(self.max_substeps, base_steps):
            raise RecipeError(
                f"{label} needs {steps} steps to keep the fastest gas ({speed:.3f} m/s) within "
                f"solver.max_cells_per_step ({self.max_cells}); solver.max_substeps is {self.max_substeps}. "
                f"Raise it, or slow the gas (emitter velocity, buoyancy, turbulence, drag)")
        return StepPlan(steps, speed)

    @staticmethod
    def grid_speed(grid) -> float:
        """The fastest face velocity component, in m/s."""
        speed = torch.zeros(1, dtype=torch.float32, device=grid.device)
        enqueue_grid_speed(grid, speed)
        return float(speed.item())

    def emitter_speed(self, start_s: float, end_s: float) -> float:
        return max((s for b, e, s in self.emitters if b < end_s and e > start_s), default=0.0)


def enqueue_grid_speed(grid, out: torch.Tensor) -> None:
    """Enqueues the device max of |u|, |v|, |w| into `out` (one float32 element) on the current stream."""
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_grid_speed", grid.info, N.field_ptr(u), N.field_ptr(v), N.field_ptr(w), N.storage_of(u),
           N.ptr(out), N.stream())


def _emitter_speed(velocity_mps, mode: str) -> float:
    velocity = np.asarray(velocity_mps, dtype=np.float64)
    if mode == "outward":
        return float(np.linalg.norm(velocity))
    return float(np.abs(velocity).max())
