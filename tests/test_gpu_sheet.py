"""Sheet assembly and the numbers file on the device against the sheet oracle (itself pinned to the
reference's sheet code, tests/test_sheet_oracle.py), on the same raw frames: the crop, margin and divisors
exactly, the packed sheet bytes exactly (at most a 1-byte difference on at most 1e-4 of the bytes is allowed:
the easing step's frame-wide sums are added in a fixed order on the device, not numpy's), the numbers text
exactly."""

import dataclasses

import numpy as np
import pytest

from oracle import sheet as S
from plume_b200.recipe.derived import derive
from plume_b200.workloads import operator_fields, plain_step_recipe

pytestmark = pytest.mark.gpu

LAYOUTS = ("heat,thickness,shade,unused", "heat,thickness,normal_x,normal_y")
BYTE_MISMATCH_SHARE = 1e-4


def rendered_frames(channels, frames=6, cells=(32, 48, 32)):
    """Raw frames of a short heat-carrying run rendered by the CUDA path (device tensor and host copy)."""
    import torch

    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper

    recipe = plain_step_recipe(cells, cycles=2, frames=frames, substeps=2)
    recipe = dataclasses.replace(recipe, output=dataclasses.replace(recipe.output, channels=channels, frame_px=64))
    derived = derive(recipe)
    d = recipe.domain
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0")
    for name, values in operator_fields(derived.cells, 4, d.ambient_k).items():
        getattr(grid, name).data.copy_(torch.from_numpy(values * (0.5 if name == "smoke" else 1.0)))
    view = sheet_domain_view(recipe, derived)
    renderer = FrameRenderer(view, recipe.render, derived.cells, channels, "cuda:0")
    stepper = Stepper(grid, recipe)
    stack = torch.empty((frames, view.height_px, view.width_px, 5), dtype=torch.float32, device="cuda:0")
    for f in range(frames):
        for n in range(derived.steps_per_frame):
            stepper.step((f * derived.steps_per_frame + n) * derived.dt_s, derived.dt_s)
        renderer.prepare(grid.smoke.data, grid.info.cell_m)
        renderer.march(grid.smoke.data, grid.temperature.data, grid.info, renderer.view_params, stack[f])
    torch.cuda.synchronize()
    return recipe, derived, view, stack, list(stack.cpu().numpy())


def compare_bytes(got, want, what):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, what
    diff = np.abs(got.astype(np.int32) - want.astype(np.int32))
    assert diff.max() <= 1, f"{what}: bytes differ by {diff.max()}"
    assert (diff > 0).mean() <= BYTE_MISMATCH_SHARE, f"{what}: {(diff > 0).mean():.2e} of bytes differ"


@pytest.mark.parametrize("channels", LAYOUTS)
@pytest.mark.parametrize("margin", [None, 0.0])
def test_device_sheet_matches_the_oracle(cuda_device, channels, margin):
    from plume_b200.sheet.assemble import assemble, pack

    recipe, derived, view, stack, host_frames = rendered_frames(channels)
    render = recipe.render if margin is None else dataclasses.replace(recipe.render, crop_margin=margin)
    assert float(stack[..., 0].max()) > 0.0  # the run glows: the heat channel is exercised
    got = assemble(stack, view, (0.0, 0.2, 0.0), recipe.output.frame_px, render, channels)
    want, crop, want_margin, heat_divisor, shade_divisor = S.assemble(host_frames, recipe.output.frame_px, render,
                                                                     channels)
    assert (got.crop.left, got.crop.top, got.crop.side) == crop
    assert got.margin == want_margin
    assert got.heat_divisor == heat_divisor and got.shade_divisor == shade_divisor
    for index, (a, b) in enumerate(zip(got.frames, want)):
        compare_bytes(a, b, f"frame {index}")
    compare_bytes(pack(got.device_frames, 4).cpu().numpy(), S.pack(want, 4), "packed sheet")


@pytest.mark.parametrize("channels", LAYOUTS)
def test_device_numbers_match_the_oracle(cuda_device, channels):
    import torch

    from plume_b200.sheet.numbers import measure

    _, derived, _, _, host_frames = rendered_frames(channels)
    want, *_ = S.assemble(host_frames, 64, plain_step_recipe().render, channels)
    rows = measure(torch.from_numpy(np.stack(want)).to("cuda:0"), derived.fps)
    for row, frame in zip(rows, want):
        coverage, box, mean_heat, mean_thick, total_thick, peak_heat = S.measure_frame(frame)
        assert row.coverage == coverage and row.box == box and row.peak_heat == peak_heat
        for a, b in ((row.mean_heat, mean_heat), (row.mean_thick, mean_thick), (row.total_thick, total_thick)):
            assert abs(a - b) <= 1e-12 * max(1.0, abs(b))
