"""Rendering smoke and temperature into a raw frame (mirrors chadmv/plume
src/plume/render/frame_renderer.py:16-94).

The sheet's channel layout picks the per-frame volume pass: the light volume for the shade layout, the
normal field for the normal layout; the other gets a one-cell stand-in. `render` copies the (H, W, 5) image
to the host; `march` writes any device image for any view (the viewer's perspective cameras).
"""

import numpy as np
import torch

from plume_b200 import _native as N
from plume_b200.recipe.schema import SHADE_LAYOUT
from plume_b200.render.light_volume import LightVolume
from plume_b200.render.normal_field import NormalField
from plume_b200.render.raw_frame import CHANNELS
from plume_b200.render.raymarch import LookParams, ViewParams


class FrameRenderer:
    def __init__(self, view, settings, cells, channels: str, device: str):
        self.device = device
        self.shade_layout = channels == SHADE_LAYOUT
        self.view_params = domain_view_params(view)
        self.look_params = _look_params(settings, self.shade_layout)
        if self.shade_layout:
            light_world = toward_light_world(view.camera, settings.light_dir)
            self.light_volume = LightVolume(cells, light_world, settings.opacity_per_density, device)
            self.light = self.light_volume.light
            self.gradient = torch.zeros((1, 1, 1, 3), dtype=torch.float32, device=device)
        else:
            self.normal_field = NormalField(cells, settings.normal_blur_cells, device)
            self.gradient = self.normal_field.gradient
            self.light = torch.zeros((1, 1, 1), dtype=torch.float32, device=device)
        self.image = torch.zeros((view.height_px, view.width_px, CHANNELS), dtype=torch.float32, device=device)
        # scratch for the marched smoke's brick map (empty-space skipping; built by every march)
        self.bricks = torch.empty(N.lib().plume_brick_floats(N.c_int3(*cells)), dtype=torch.float32, device=device)
        self._host = torch.empty(self.image.shape, dtype=torch.float32, pin_memory=True)
        self._side = None  # render_async's stream, snapshot and last completion event
        self._snapshot = None
        self._last_done = None

    def render(self, grid) -> np.ndarray:
        return self.render_fields(grid.smoke.data, grid.temperature.data, grid.info)

    def render_async(self, grid) -> "PendingFrame":
        """render(grid) overlapped with what the caller enqueues next (no reference counterpart). Smoke and
        temperature are copied to a snapshot on the caller's stream; the volume pass, the march and the copy
        to pinned host memory then run on the renderer's own stream, so the caller's next substeps may
        overwrite the grid at once. PendingFrame.result() waits for the frame. Frames of one renderer complete
        in order; a new snapshot waits for the previous frame's march."""
        main = torch.cuda.current_stream()
        smoke, temperature = grid.smoke.data, grid.temperature.data
        if self._side is None:
            self._side = torch.cuda.Stream(device=smoke.device)
        if self._snapshot is None or self._snapshot[0].shape != smoke.shape or self._snapshot[0].dtype != smoke.dtype:
            self._snapshot = (torch.empty_like(smoke), torch.empty_like(temperature))
        if self._last_done is not None:
            main.wait_event(self._last_done)
        self._snapshot[0].copy_(smoke)
        self._snapshot[1].copy_(temperature)
        ready = torch.cuda.Event()
        ready.record(main)
        host = torch.empty(self.image.shape, dtype=torch.float32, pin_memory=True)
        with torch.cuda.stream(self._side):
            self._side.wait_event(ready)
            self.prepare(self._snapshot[0], grid.info.cell_m)
            self.march(self._snapshot[0], self._snapshot[1], grid.info, self.view_params, self.image)
            host.copy_(self.image, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self._side)
        self._last_done = done
        return PendingFrame(done, host)

    def wait_for(self, stream=None) -> None:
        """Makes `stream` (the current stream by default) wait for every frame render_async has enqueued."""
        if self._last_done is not None:
            (stream or torch.cuda.current_stream()).wait_event(self._last_done)

    def render_fields(self, smoke, temperature, info) -> np.ndarray:
        """The raw frame of these fields over the domain view, copied to the host."""
        self.wait_for()  # frames render_async has in flight use the same scratch
        self.prepare(smoke, info.cell_m)
        self.march(smoke, temperature, info, self.view_params, self.image)
        self._host.copy_(self.image, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self._host.numpy().copy()

    def prepare(self, smoke, cell_m: float) -> None:
        """The volume pass for marches of this same smoke. In the shade layout only the light at the cells such
        a march reads is computed (the rest hold 1); those cells match LightVolume.compute bit for bit."""
        if self.shade_layout:
            self.light = self.light_volume.compute(smoke, cell_m, march_cells=True)
        else:
            self.gradient = self.normal_field.compute(smoke)

    def march(self, smoke, temperature, info, view: ViewParams, image) -> None:
        """Marches `image` for `view` through the fields, with the volume pass of the last prepare."""
        gradient_shape = N.c_int3(*self.gradient.shape[:3])
        bricks = N.ptr(self.bricks) if tuple(self.bricks.shape) == (N.lib().plume_brick_floats(N.shape3(smoke)),) \
            else None
        if temperature.dtype != smoke.dtype:
            raise TypeError("smoke and temperature must have the same storage type")
        N.call("plume_raymarch", info, N.field_ptr(smoke), N.field_ptr(temperature), N.storage_of(smoke),
               N.ptr(self.gradient), gradient_shape,
               N.ptr(self.light), N.shape3(self.light), view, self.look_params, N.ptr(image), image.shape[0],
               image.shape[1], bricks, N.stream())


class PendingFrame:
    """A frame FrameRenderer.render_async has enqueued: result() waits for it and returns the (H, W, 5) array."""

    def __init__(self, done, host):
        self._done = done
        self._host = host

    def result(self) -> np.ndarray:
        self._done.synchronize()
        return self._host.numpy().copy()


def toward_light_world(camera, light_dir) -> np.ndarray:
    x, y, z = light_dir
    return x * camera.right + y * camera.up + z * camera.toward


def domain_view_params(view) -> ViewParams:
    params = ViewParams()
    params.right = N.f3(view.camera.right)
    params.up = N.f3(view.camera.up)
    params.toward = N.f3(view.camera.toward)
    params.left_m, params.top_m, params.pixel_m = view.left_m, view.top_m, view.pixel_m
    params.perspective = 0
    params.eye = N.f3((0.0, 0.0, 0.0))
    return params


def _look_params(settings, shade_layout: bool) -> LookParams:
    params = LookParams()
    params.opacity_per_density = settings.opacity_per_density
    params.glow_start_k = settings.glow_start_k
    params.smoke_hides_heat = settings.smoke_hides_heat
    params.normal_fade_thickness = settings.normal_fade_thickness
    params.shade_layout = 1 if shade_layout else 0
    params.shade_fill = settings.shade_fill
    return params
