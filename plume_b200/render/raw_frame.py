"""Raw frame channel layout (chadmv/plume src/plume/render/raw_frame.py:15-29): (height, width, 5) float32 with
heat, thickness, then normal x/y/z (normal layout) or shade*thickness and two zeros (shade layout)."""

import numpy as np

from plume_b200.recipe.schema import NORMAL_LAYOUT

HEAT = 0
THICKNESS = 1
NORMAL_X = 2
NORMAL_Y = 3
NORMAL_Z = 4
SHADE = 2
CHANNELS = 5


def empty_pixel(channels: str) -> np.ndarray:
    pixel = np.zeros(CHANNELS, dtype=np.float32)
    if channels == NORMAL_LAYOUT:
        pixel[NORMAL_Z] = 1.0
    return pixel
