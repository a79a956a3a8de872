"""A live run (mirrors chadmv/plume src/plume/view/live_run.py): the recipe's simulation advanced one frame at a
time, each frame captured exactly as `plume run` captures it (the sheet camera's raw frame through the same
FrameRenderer), its smoke, temperature and centred velocity kept in the frame cache for drawing from any
angle, and the faces its smoke reached noted for the numbers strip. When the last frame lands the sheet is
assembled (on the device, at once: the reference assembles on a worker thread with host numpy) for its heat
and shade divisors and crop. A re-capture renders a finished run's kept frames again with new render
settings instead of simulating.

The window itself is out of scope; this is the headless part the window drives."""

import itertools
import math
import time

import numpy as np
import torch

from plume_b200 import _native as N
from plume_b200.render.camera import sheet_domain_view
from plume_b200.render.frame_renderer import FrameRenderer
from plume_b200.render.raw_frame import HEAT
from plume_b200.run import seat_point
from plume_b200.sheet.assemble import assemble
from plume_b200.sim.run import simulate_frames
from plume_b200.view.frame_cache import FrameCache, narrow, widen  # noqa: F401  (the casts live with the cache)

_SERIALS = itertools.count(1)
FACE_NAMES = ("left", "right", "bottom", "top", "back", "front")  # x low, x high, y low, y high, z low, z high
CEILING = "top"


def boundary_layers(smoke: torch.Tensor) -> torch.Tensor:
    """(6, S, S) with S the largest dimension: layers[face, a, b], a and b the face's other axes in x, y, z
    order, 0 past the face's size (live_run.py:42-57)."""
    side = max(smoke.shape)
    layers = torch.empty((6, side, side), dtype=torch.float32, device=smoke.device)
    N.call("plume_view_boundary_layers", N.ptr(smoke), N.shape3(smoke), N.ptr(layers), N.stream())
    return layers


def visible_density(recipe) -> float:
    """Smoke density at which one cell's opacity reaches one byte step (1/255)."""
    return -math.log(1.0 - 1.0 / 255.0) / (recipe.render.opacity_per_density * recipe.domain.cell_m)


def faces_reached(layers: np.ndarray, recipe) -> tuple:
    """The open faces, and the ceiling, whose boundary layer holds visible smoke, in FACE_NAMES order."""
    largest = layers.reshape(len(FACE_NAMES), -1).max(axis=1)
    threshold = visible_density(recipe)
    faces = recipe.domain.faces
    return tuple(name for name, value in zip(FACE_NAMES, largest, strict=True)
                 if value >= threshold and (name == CEILING or getattr(faces, name) == "open"))


class LiveRun:
    """One run of a resolved recipe; call `advance` once per window update while it is `capturing`."""

    def __init__(self, recipe, derived, device: str, budget_bytes: float, shared_with_compare: bool = False,
                 source: "LiveRun | None" = None):
        self.serial = next(_SERIALS)
        self.recipe = recipe
        self.derived = derived
        self.device = device
        self.view = sheet_domain_view(recipe, derived)
        self.renderer = FrameRenderer(self.view, recipe.render, derived.cells, recipe.output.channels, device)
        self.recaptured = source is not None
        self.source = source
        self.raw_frames = []
        self.assembled = None
        self.assembly_error = None
        self.started_s = time.perf_counter()
        self.stopped = False
        self._largest_raw_heat = 0.0
        if source is None:
            self.simulation_serial = self.serial
            self.cache = FrameCache(derived.cells, recipe.time.frames, budget_bytes, device, shared_with_compare)
            self.info = None
            self.steps = None
            self.elapsed_s = 0.0
            self.edges = {}
            self._frames = simulate_frames(recipe, derived, device)
        else:
            self.simulation_serial = source.simulation_serial
            self.cache = source.cache
            self.info = source.info
            self.steps = source.steps
            self.elapsed_s = source.elapsed_s
            self.edges = source.edges
            self._frames = self._recaptured_frames()

    @classmethod
    def recapture(cls, source: "LiveRun", recipe) -> "LiveRun":
        """A run of `recipe` (the same simulation stage) over a finished source run's kept frames."""
        if not source.can_recapture():
            raise ValueError("a re-capture needs a finished run that kept every frame")
        if source.recaptured and source.capturing and source.source is not None:
            source = source.source
        return cls(recipe, source.derived, source.device, 0.0, source=source)

    def can_recapture(self) -> bool:
        return self.done and not self.cache.thinned

    @property
    def capturing(self) -> bool:
        return not self.stopped and self.landed < self.frames

    @property
    def frames(self) -> int:
        return self.recipe.time.frames

    @property
    def landed(self) -> int:
        return len(self.raw_frames)

    @property
    def done(self) -> bool:
        return self.steps is not None

    def advance(self):
        """Simulates (or re-captures) and captures the next frame and returns its index; None once every
        frame is captured or the run stopped."""
        if not self.capturing:
            return None
        if self.recaptured:
            return next(self._frames)
        frame, grid = next(self._frames)
        if self.info is None:
            self.info = grid.info
        self._keep_raw(self.renderer.render(grid))
        self.cache.store(frame, grid.smoke.data, grid.temperature.data,
                         tuple(field.data for field in grid.velocity_fields()))
        self.edges[frame] = faces_reached(boundary_layers(grid.smoke.data).cpu().numpy(), self.recipe)
        if frame == self.frames - 1:
            self._finish()
        return frame

    def _keep_raw(self, raw: np.ndarray) -> None:
        self.raw_frames.append(raw)
        self._largest_raw_heat = max(self._largest_raw_heat, float(raw[..., HEAT].max()))

    def _recaptured_frames(self):
        scratch = self.cache.scratch()
        for frame in range(self.frames):
            smoke, temperature = self.cache.load(frame, scratch)
            self._keep_raw(self.renderer.render_fields(smoke, temperature, self.info))
            if frame == self.frames - 1:
                self._assemble()
            yield frame

    def cancel(self) -> None:
        """Stops the run where it is; its frames stay drawable."""
        if self.capturing:
            self.stopped = True
            if not self.recaptured:
                self.elapsed_s = time.perf_counter() - self.started_s
        self._frames.close()

    def poll_assembly(self) -> bool:
        """True once the sheet is assembled (at once here: the device assembles as the last frame lands)."""
        return self.assembled is not None or self.assembly_error is not None

    def wait_for_assembly(self) -> None:
        """Nothing to wait for: kept for the window's and the tests' calling pattern."""

    @property
    def heat_divisor(self) -> float:
        """What heat 1 means: the sheet's divisor once assembled, else a re-capture's source's, else the
        largest raw heat so far."""
        if self.assembled is None and self.source is not None:
            return self.source.heat_divisor
        divisor = self.assembled.heat_divisor if self.assembled else self._largest_raw_heat
        return divisor if divisor > 0.0 else 1.0

    @property
    def shade_divisor(self) -> float:
        if self.assembled is None and self.source is not None:
            return self.source.shade_divisor
        if self.assembled is None or self.assembled.shade_divisor is None:
            return 1.0
        return self.assembled.shade_divisor

    def _finish(self) -> None:
        try:
            next(self._frames)
        except StopIteration as finished:
            self.steps = finished.value
        self.elapsed_s = time.perf_counter() - self.started_s
        self._assemble()

    def _assemble(self) -> None:
        try:
            self.assembled = assemble(list(self.raw_frames), self.view, seat_point(self.recipe),
                                      self.recipe.output.frame_px, self.recipe.render, self.recipe.output.channels,
                                      self.device)
        except Exception as error:  # noqa: BLE001 - reported in the status line; the run stays drawable
            self.assembly_error = f"sheet assembly failed: {error}"
        else:
            self.source = None
