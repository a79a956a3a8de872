"""The `plume run` pipeline on the device (mirrors chadmv/plume src/plume/cli/run.py:44-127): simulate with each
frame rendered into one device stack, assemble the sheet on the device and measure its numbers there. The
reference also writes the PNG sheets, the sheet JSON and the settings file; those stay with the caller, who
gets the packed sheet, the assembled frames and the numbers text."""

from dataclasses import dataclass

import numpy as np
import torch

from plume_b200.recipe.derived import derive
from plume_b200.render.camera import sheet_domain_view
from plume_b200.render.frame_renderer import FrameRenderer
from plume_b200.render.raw_frame import CHANNELS
from plume_b200.sheet.assemble import AssembledFrames, assemble, pack
from plume_b200.sheet.numbers import RunFacts, measure, numbers_text
from plume_b200.sim.run import StepLog, simulate


@dataclass(frozen=True)
class DeviceRun:
    recipe: object
    derived: object
    view: object
    raw: torch.Tensor            # (frames, H, W, 5) raw frames
    assembled: AssembledFrames   # quantised frames (host and device copies), crop, divisors, seat
    sheet: torch.Tensor          # the packed (rows * size, columns * size, 4) sheet
    numbers: str                 # the numbers file's text
    steps: StepLog


def seat_point(recipe) -> np.ndarray:
    """The world point the sheet's seat marks: the centre of the emitter camera.seat names
    (sheet/assemble.py:63-66)."""
    emitter = next(e for e in recipe.emitter if e.name == recipe.camera.seat)
    return np.array(emitter.center_m, dtype=np.float64)


def run_recipe(recipe, source: str, device: str = "cuda:0") -> DeviceRun:
    """Runs a loaded recipe end to end on `device`; `source` is the recipe path the numbers file names."""
    derived = derive(recipe)
    view = sheet_domain_view(recipe, derived)
    channels = recipe.output.channels
    renderer = FrameRenderer(view, recipe.render, derived.cells, channels, device)
    raw = torch.empty((recipe.time.frames, view.height_px, view.width_px, CHANNELS), dtype=torch.float32,
                      device=device)

    def capture(frame, grid):
        renderer.prepare(grid.smoke.data, grid.info.cell_m)
        renderer.march(grid.smoke.data, grid.temperature.data, grid.info, renderer.view_params, raw[frame])

    steps = simulate(recipe, derived, device, capture)
    assembled = assemble(raw, view, seat_point(recipe), recipe.output.frame_px, recipe.render, channels, device)
    nx, ny, nz = derived.cells
    facts = RunFacts(recipe=source, backend=device, grid=f"{nx} x {ny} x {nz} cells of {recipe.domain.cell_m:.6f} m",
                     fps=derived.fps, frame_m=assembled.frame_m, heat_divisor=assembled.heat_divisor,
                     channels=channels, shade_divisor=assembled.shade_divisor)
    numbers = numbers_text(measure(assembled.device_frames, derived.fps), facts)
    return DeviceRun(recipe, derived, view, raw, assembled, pack(assembled.device_frames, recipe.output.columns),
                     numbers, steps)
