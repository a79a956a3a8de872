"""The viewer oracle's look matches the host composite a game's shader is to match (the reference's own
check, tests/view/test_viewport.py:47-72: within one byte), and its composite is the reference's
(report/composite.py, when the reference is mounted); the product's colour tables are the reference's."""

import itertools
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import view as V
from plume_b200.recipe.schema import LookSettings
from plume_b200.view.color import hex_to_linear, ramp, to_srgb_bytes

BYTES = np.arange(0, 256, 15, dtype=np.uint8)
HEAT_DIVISOR, SHADE_DIVISOR = 7.3, 0.8
BACKGROUND = "#aac476"
LIGHT_DIR = (0.5, 0.8, 0.3)
REFERENCE = Path(os.environ.get("PLUME_REFERENCE", "/root/reference")) / "src"


def byte_grid(shade: bool) -> np.ndarray:
    if shade:
        rows = [(h, g, b, 255) for h, g, b in itertools.product(BYTES, BYTES, BYTES)]
    else:
        rows = [(h, g, b, a) for h, g, b, a in itertools.product(BYTES, BYTES, BYTES, BYTES)
                if (b / 255 * 2 - 1) ** 2 + (a / 255 * 2 - 1) ** 2 <= 1.0]
    return np.array(rows, dtype=np.uint8)[None, :, :]


def raw_from_pixels(rgba: np.ndarray, shade: bool) -> np.ndarray:
    values = rgba.astype(np.float64) / 255.0
    raw = np.zeros((*rgba.shape[:2], 5), dtype=np.float64)
    raw[..., 0] = values[..., 0] * HEAT_DIVISOR
    raw[..., 1] = values[..., 1]
    if shade:
        raw[..., 2] = values[..., 2] * SHADE_DIVISOR * values[..., 1]
    else:
        nx, ny = values[..., 2] * 2.0 - 1.0, values[..., 3] * 2.0 - 1.0
        raw[..., 2], raw[..., 3], raw[..., 4] = nx, ny, np.sqrt(np.maximum(0.0, 1.0 - nx**2 - ny**2))
    return raw


def tables(look: LookSettings):
    positions = np.linspace(0.0, 1.0, 1024)
    return (ramp(look.smoke_ramp, positions).astype(np.float32), ramp(look.emission_ramp, positions).astype(np.float32),
            to_srgb_bytes(np.linspace(0.0, 1.0, 16384)))


@pytest.mark.parametrize("shade", [True, False])
def test_oracle_look_matches_the_composite_within_a_byte(shade):
    look = LookSettings()
    rgba = byte_grid(shade)
    raw = raw_from_pixels(rgba, shade)
    smoke_ramp, emission_ramp, srgb = tables(look)
    toward = np.array(LIGHT_DIR) / np.linalg.norm(LIGHT_DIR)

    def viewer(view):
        return V.look(raw, smoke_ramp, emission_ramp, srgb, view, shade, HEAT_DIVISOR, SHADE_DIVISOR,
                      look.shade_depth, look.ambient, toward, hex_to_linear(BACKGROUND)).astype(int)

    expected = to_srgb_bytes(V.composite(rgba, hex_to_linear(BACKGROUND), shade, look, LIGHT_DIR, ramp)).astype(int)
    assert np.abs(viewer(0)[..., :3] - expected).max() <= 1
    assert np.array_equal(viewer(1)[..., 0], rgba[..., 0])
    assert np.array_equal(viewer(2)[..., 1], rgba[..., 1])


@pytest.mark.skipif(not (REFERENCE / "plume").exists(), reason="the reference is not mounted")
def test_oracle_composite_and_colour_tables_are_the_references():
    import sys

    sys.path.insert(0, str(REFERENCE))
    from plume.recipe.schema import LookSettings as RefLook
    from plume.report import color as ref_color
    from plume.report.composite import SheetLook, composite

    look = LookSettings()
    assert RefLook().smoke_ramp == look.smoke_ramp and RefLook().emission_ramp == look.emission_ramp
    assert (RefLook().ambient, RefLook().shade_depth) == (look.ambient, look.shade_depth)
    positions = np.linspace(0.0, 1.0, 1024)
    assert np.array_equal(ref_color.ramp(RefLook().smoke_ramp, positions), ramp(look.smoke_ramp, positions))
    assert np.array_equal(ref_color.to_srgb_bytes(positions), to_srgb_bytes(positions))
    for shade, channels in ((True, "heat,thickness,shade,unused"), (False, "heat,thickness,normal_x,normal_y")):
        rgba = byte_grid(shade)
        want = composite(rgba, BACKGROUND, SheetLook(look=RefLook(), channels=channels, light_dir=LIGHT_DIR))
        got = V.composite(rgba, hex_to_linear(BACKGROUND), shade, look, LIGHT_DIR, ramp)
        assert np.array_equal(got, want)
