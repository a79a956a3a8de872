"""The Volume view's device steps after the march (mirrors chadmv/plume src/plume/view/viewport.py:78-190):
the look (a raw march image to display bytes by view) and the centre ray's depth.

Look: the contact sheets' composite over a background, in sRGB, with the smoke and emission ramps and the sRGB
curve tabulated from the colour helpers; Heat, Thickness, Shade: the channel as a gray byte; the normal
layout's fourth view shows (n + 1) / 2 as RGB. Heat is divided by the run's heat divisor and the shade by its
shade divisor, as the sheet's are.
"""

import numpy as np
import torch

from plume_b200 import _native as N
from plume_b200.recipe.schema import SHADE_LAYOUT
from plume_b200.render.raymarch import FAR_M
from plume_b200.view.color import hex_to_linear, ramp, to_srgb_bytes

LOOK, HEAT_VIEW, THICKNESS_VIEW, SHADE_VIEW = 0, 1, 2, 3
RAMP_TABLE_SIZE = 1024
SRGB_TABLE_SIZE = 16384
RELEASE_THICKNESS = 0.5


class LookTables:
    """The composite's ramps and sRGB curve on the device."""

    def __init__(self, recipe, device: str):
        positions = np.linspace(0.0, 1.0, RAMP_TABLE_SIZE)
        self.smoke_ramp = torch.from_numpy(ramp(recipe.look.smoke_ramp, positions).astype(np.float32)).to(device)
        self.emission_ramp = torch.from_numpy(ramp(recipe.look.emission_ramp, positions).astype(np.float32)).to(device)
        self.srgb = torch.from_numpy(to_srgb_bytes(np.linspace(0.0, 1.0, SRGB_TABLE_SIZE))).to(device)


def look_inputs(recipe, view: int, heat_divisor: float, shade_divisor: float, background_hex: str,
                toward_light_camera) -> N.PlumeLookInputs:
    inputs = N.PlumeLookInputs()
    inputs.view = view
    inputs.shade_layout = 1 if recipe.output.channels == SHADE_LAYOUT else 0
    inputs.heat_divisor = heat_divisor if heat_divisor > 0.0 else 1.0
    inputs.shade_divisor = shade_divisor if shade_divisor > 0.0 else 1.0
    inputs.shade_depth = recipe.look.shade_depth
    inputs.ambient = recipe.look.ambient
    inputs.toward_light = N.f3(toward_light_camera)
    inputs.background = N.f3(hex_to_linear(background_hex))
    return inputs


def launch_look(raw: torch.Tensor, tables: LookTables, inputs, out: torch.Tensor) -> None:
    """A raw march image ((height, width, 5) float32, device) into display bytes ((height, width, 4) uint8)."""
    height, width = raw.shape[0], raw.shape[1]
    N.call("plume_view_look", N.ptr(raw), height, width, N.ptr(tables.smoke_ramp), N.ptr(tables.emission_ramp),
           tables.smoke_ramp.shape[0], N.ptr(tables.srgb, torch.uint8), tables.srgb.shape[0], inputs,
           N.ptr(out, torch.uint8), N.stream())


def look_bytes(raw: np.ndarray, tables: LookTables, inputs, device: str) -> np.ndarray:
    """The look over a host raw image: (height, width, 4) uint8."""
    image = torch.from_numpy(np.ascontiguousarray(raw, dtype=np.float32)).to(device)
    out = torch.zeros((*raw.shape[:2], 4), dtype=torch.uint8, device=device)
    launch_look(image, tables, inputs, out)
    return out.cpu().numpy()


def center_depth(smoke: torch.Tensor, info, origin, direction, opacity_per_density: float,
                 threshold: float = RELEASE_THICKNESS) -> float:
    """The distance along the ray at which the march's thickness first reaches `threshold`; -1 if never."""
    result = torch.empty(1, dtype=torch.float32, device=smoke.device)
    N.call("plume_view_center_depth", N.ptr(smoke), info, N.f3(origin), N.f3(direction), opacity_per_density,
           threshold, N.ptr(result), N.stream())
    return float(result.item())


def center_ray(camera):
    """The view's centre ray: (origin, direction) (viewport.py:222-232)."""
    direction = -np.asarray(camera.toward, dtype=np.float64)
    if camera.perspective:
        return np.asarray(camera.eye, dtype=np.float64), direction
    center_x = camera.left + camera.pixel * camera.width_px / 2
    center_y = camera.top - camera.pixel * camera.height_px / 2
    origin = (np.asarray(camera.right) * center_x + np.asarray(camera.up) * center_y
              + np.asarray(camera.toward) * FAR_M)
    return origin, direction
