"""Many independent recipes on one GPU: the batched form of the frame loop (sim/run.py) for preview variants
and parameter sweeps of uneven grid sizes.

Each instance keeps its own grid, stepper, CFL cap and CUDA stream. A host scheduler walks every instance
through the same blocks run.py walks one through (warmup blocks, then one block per frame): it enqueues the
block's fastest-speed reduction and a 4-byte copy into pinned memory behind the instance's previous block,
and when that copy has landed (an event query, no device-wide synchronisation) plans the block with the
instance's StepCap and enqueues its substeps. Instances therefore never wait for one another, and the
kernels of different instances -- most of them far too small to fill the GPU alone, such as the multigrid's
coarse levels -- run side by side on the GPU. Each substep is one plume_step call (its pressure solve one
CUDA-graph replay), so the results are those of running each recipe alone through simulate_frames.
"""

from collections.abc import Callable, Sequence
from dataclasses import dataclass, field

import torch

from plume_b200.recipe.derived import derive
from plume_b200.sim.grid import Grid, make_grid
from plume_b200.sim.run import StepLog
from plume_b200.sim.step_cap import StepCap, enqueue_grid_speed
from plume_b200.sim.stepper import Stepper

# capture(instance index, frame index, grid): called on the instance's stream after the frame's substeps
BatchCapture = Callable[[int, int, Grid], None]


@dataclass
class _Block:
    base_steps: int
    label: str
    frame: int | None  # None for a warmup block


@dataclass
class _Instance:
    recipe: object
    derived: object
    grid: Grid
    stepper: Stepper
    cap: StepCap
    stream: torch.cuda.Stream
    blocks: list
    speed: torch.Tensor            # device float, the block's fastest face speed
    host_speed: torch.Tensor       # pinned copy
    ready: torch.cuda.Event | None = None
    next_block: int = 0
    base_done: int = 0
    warmup_steps: int = 0
    frame_steps: list = field(default_factory=list)

    @property
    def done(self) -> bool:
        return self.next_block >= len(self.blocks)


def _blocks(recipe, derived) -> list:
    blocks, remaining = [], derived.warmup_steps
    while remaining > 0:
        size = min(remaining, derived.steps_per_frame)
        blocks.append(_Block(size, "warmup", None))
        remaining -= size
    blocks += [_Block(derived.steps_per_frame, f"frame {f}", f) for f in range(recipe.time.frames)]
    return blocks


class Batch:
    """Steps many recipes through their whole runs on one device, concurrently."""

    def __init__(self, recipes: Sequence, device: str, storage=torch.float32, initial_state=None):
        """`initial_state(index, grid)`, when given, fills an instance's fields before its first block (on the
        current stream)."""
        self.device = device
        self.initial_state = initial_state
        self.instances: list[_Instance] = []
        current = torch.cuda.current_stream(device)
        for index, recipe in enumerate(recipes):
            derived = derive(recipe)
            d = recipe.domain
            grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device, storage=storage)
            if initial_state is not None:
                initial_state(index, grid)
            # Everything that fills device memory on the current stream (the grid, the stepper's multigrid
            # levels and scratch, the speed slot) is enqueued before the instance's stream waits on it.
            stepper = Stepper(grid, recipe)
            speed = torch.zeros(1, dtype=torch.float32, device=device)
            host_speed = torch.zeros(1, dtype=torch.float32, pin_memory=True)
            stream = torch.cuda.Stream(device)
            stream.wait_stream(current)
            self.instances.append(_Instance(
                recipe=recipe, derived=derived, grid=grid, stepper=stepper, cap=StepCap(recipe),
                stream=stream, blocks=_blocks(recipe, derived), speed=speed, host_speed=host_speed))

    def _request_speed(self, inst: _Instance) -> None:
        with torch.cuda.stream(inst.stream):
            enqueue_grid_speed(inst.grid, inst.speed)
            inst.host_speed.copy_(inst.speed, non_blocking=True)
            inst.ready = torch.cuda.Event()
            inst.ready.record(inst.stream)

    def _run_block(self, index: int, inst: _Instance, capture: BatchCapture | None) -> None:
        block = inst.blocks[inst.next_block]
        dt = inst.derived.dt_s
        start_s, length_s = inst.base_done * dt, block.base_steps * dt
        steps = inst.cap.plan_for_speed(float(inst.host_speed[0]), start_s, length_s, block.base_steps,
                                        block.label).steps
        with torch.cuda.stream(inst.stream):
            for n in range(steps):
                if steps == block.base_steps:
                    inst.stepper.step((inst.base_done + n) * dt, dt)
                else:
                    inst.stepper.step(start_s + n * length_s / steps, length_s / steps)
            if block.frame is None:
                inst.warmup_steps += steps
            else:
                inst.frame_steps.append(steps)
                if capture is not None:
                    capture(index, block.frame, inst.grid)
        inst.base_done += block.base_steps
        inst.next_block += 1
        inst.ready = None

    def reset(self) -> None:
        """Puts every instance back at its start (fields and pressure zero, temperature ambient, then
        `initial_state`), keeping its arrays, so that a second run repeats the first with the allocations and
        the pressure solves' CUDA graphs already in place."""
        current = torch.cuda.current_stream(self.device)
        for inst in self.instances:
            current.wait_stream(inst.stream)
        for index, inst in enumerate(self.instances):
            grid = inst.grid
            for field in (*grid.velocity_fields(), grid.smoke, grid.temperature):
                for array in (field.data, field.hat, field.next):
                    array.zero_()
            for array in (grid.temperature.data, grid.temperature.hat, grid.temperature.next):
                array.fill_(inst.recipe.domain.ambient_k)
            grid.pressure.zero_()
            grid.divergence.zero_()
            if self.initial_state is not None:
                self.initial_state(index, grid)
            inst.next_block, inst.base_done, inst.warmup_steps, inst.ready = 0, 0, 0, None
            inst.frame_steps = []
        for inst in self.instances:
            inst.stream.wait_stream(current)

    def run(self, capture: BatchCapture | None = None, sequential: bool = False) -> list[StepLog]:
        """Runs every instance to its last frame; returns each instance's StepLog (run.py's record). With
        `sequential` the instances run one after another, each to its end before the next starts (the plain
        one-at-a-time schedule on the same arrays)."""
        if sequential:
            for index, inst in enumerate(self.instances):
                while not inst.done:
                    self._request_speed(inst)
                    inst.ready.synchronize()
                    self._run_block(index, inst, capture)
            return self._logs()
        for inst in self.instances:
            if not inst.done:
                self._request_speed(inst)
        active = [(i, inst) for i, inst in enumerate(self.instances) if not inst.done]
        while active:
            progressed = False
            for index, inst in active:
                if inst.ready is not None and inst.ready.query():
                    self._run_block(index, inst, capture)
                    if not inst.done:
                        self._request_speed(inst)
                    progressed = True
            active = [(i, inst) for i, inst in active if not inst.done]
            if not progressed and active:
                active[0][1].ready.synchronize()  # nothing landed yet: wait for the oldest request
        return self._logs()

    def _logs(self) -> list[StepLog]:
        for inst in self.instances:
            torch.cuda.current_stream(self.device).wait_stream(inst.stream)
        return [StepLog(inst.warmup_steps, tuple(inst.frame_steps), inst.derived.steps_per_frame,
                        inst.derived.warmup_steps) for inst in self.instances]

    @property
    def grids(self) -> list[Grid]:
        return [inst.grid for inst in self.instances]


def run_one_at_a_time(recipes: Sequence, device: str, storage=torch.float32, initial_state=None,
                      capture: BatchCapture | None = None) -> list[StepLog]:
    """The plain schedule: each recipe's whole run through simulate_frames, one after another."""
    from plume_b200.sim.run import simulate_frames

    logs = []
    for index, recipe in enumerate(recipes):
        derived = derive(recipe)
        frames = simulate_frames(recipe, derived, device, storage=storage,
                                 initial_state=None if initial_state is None else
                                 (lambda grid, index=index: initial_state(index, grid)))
        while True:
            try:
                frame, grid = next(frames)
            except StopIteration as finished:
                logs.append(finished.value)
                break
            if capture is not None:
                capture(index, frame, grid)
    return logs
