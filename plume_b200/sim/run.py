"""The frame loop (mirrors chadmv/plume src/plume/sim/run.py:22-85).

Warmup runs in blocks of the frame's base step count (the last one shorter); each frame is one block. A
block starts at `base steps so far * dt`, so the clock never drifts, and the CFL cap may split it into more,
shorter steps. The generator yields the live grid after each frame's steps.
"""

from collections.abc import Callable, Generator
from dataclasses import dataclass

from plume_b200.sim.grid import Grid, make_grid
from plume_b200.sim.step_cap import StepCap
from plume_b200.sim.stepper import Stepper

Capture = Callable[[int, Grid], None]


@dataclass(frozen=True)
class StepLog:
    warmup_steps: int
    steps_per_frame: tuple
    base_steps_per_frame: int
    base_warmup_steps: int

    @property
    def total_steps(self) -> int:
        return self.warmup_steps + sum(self.steps_per_frame)

    @property
    def added_steps(self) -> int:
        base = self.base_warmup_steps + self.base_steps_per_frame * len(self.steps_per_frame)
        return self.total_steps - base


def simulate(recipe, derived, device: str, capture: Capture) -> StepLog:
    """Runs the whole recipe, calling capture(frame_index, grid) once per frame, in order."""
    frames = simulate_frames(recipe, derived, device)
    while True:
        try:
            frame, grid = next(frames)
        except StopIteration as finished:
            return finished.value
        capture(frame, grid)


def simulate_frames(recipe, derived, device: str, storage=None,
                    initial_state=None) -> Generator[tuple[int, Grid], None, StepLog]:
    """`storage` (float32 by default; bfloat16 or float16 for the mixed-precision step) and
    `initial_state(grid)` (fills the fields before the first step) extend the reference's signature."""
    import torch

    grid = make_grid(derived, recipe.domain.cell_m, recipe.domain.faces, recipe.domain.ambient_k, device,
                     storage=torch.float32 if storage is None else storage)
    if initial_state is not None:
        initial_state(grid)
    stepper = Stepper(grid, recipe)
    cap = StepCap(recipe)
    base_done = 0

    def run_block(base_steps: int, label: str) -> int:
        nonlocal base_done
        start_s = base_done * derived.dt_s
        length_s = base_steps * derived.dt_s
        steps = cap.plan(grid, start_s, length_s, base_steps, label).steps
        for index in range(steps):
            if steps == base_steps:
                stepper.step((base_done + index) * derived.dt_s, derived.dt_s)
            else:
                stepper.step(start_s + index * length_s / steps, length_s / steps)
        base_done += base_steps
        return steps

    warmup_steps = 0
    remaining = derived.warmup_steps
    while remaining > 0:
        block = min(remaining, derived.steps_per_frame)
        warmup_steps += run_block(block, "warmup")
        remaining -= block
    frame_steps = []
    for frame in range(recipe.time.frames):
        frame_steps.append(run_block(derived.steps_per_frame, f"frame {frame}"))
        yield frame, grid
    return StepLog(warmup_steps, tuple(frame_steps), derived.steps_per_frame, derived.warmup_steps)
