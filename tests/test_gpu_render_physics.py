"""The reference's render property tests (tests/render/test_raymarch.py, test_shade.py, test_view_cameras.py in
chadmv/plume), run on the CUDA path: Beer-Lambert attenuation of a uniform slab, sphere normals, heat hidden
by smoke, the orientation of a top-down view, shading by the light volume, and the perspective camera."""

import math

import numpy as np
import pytest

from plume_b200.recipe.schema import NORMAL_LAYOUT, SHADE_LAYOUT, RenderSettings
from plume_b200.render.camera import make_camera, make_domain_view
from plume_b200.render.raw_frame import CHANNELS, HEAT, NORMAL_X, NORMAL_Y, NORMAL_Z, SHADE, THICKNESS
from support import blob, cuda_grid, host, put

pytestmark = pytest.mark.gpu

CELL_M = 0.1
CELLS = (16, 16, 16)
LEFT = (-1.0, 0.0, 0.0)


def grid16():
    return cuda_grid(cells=CELLS, cell_m=CELL_M)


def box_view(elevation_deg=0.0, azimuth_deg=0.0):
    """The 1.6 m box's domain view at 2 px per cell: 32 x 32 px."""
    return make_domain_view(make_camera(elevation_deg, azimuth_deg), (-0.8, 0.0, -0.8), (1.6, 1.6, 1.6), CELL_M, 2.0)


def render(grid, elevation_deg=0.0, channels=NORMAL_LAYOUT, **settings):
    from plume_b200.render.frame_renderer import FrameRenderer

    view = box_view(elevation_deg)
    return view, FrameRenderer(view, RenderSettings(**settings), grid.cells, channels, "cuda:0").render(grid)


def sphere(grid):
    put(grid.smoke.data, 3.0 * (blob(CELLS, (8.0, 8.0, 8.0), 3.0) > 0.3))
    return grid


# ---- the march (render/test_raymarch.py) --------------------------------------------------------------------

def test_the_domain_view_covers_the_box_at_two_pixels_per_cell():
    view = box_view()
    assert (view.width_px, view.height_px) == (32, 32)
    assert view.to_pixels(np.array([-0.8, 1.6, 0.0])) == pytest.approx((0.0, 0.0))


def test_a_uniform_slab_follows_beer_lambert(cuda_device):
    grid = grid16()
    grid.smoke.data.fill_(0.5)
    _, image = render(grid, opacity_per_density=2.0)
    assert image[16, 16, THICKNESS] == pytest.approx(1.0 - math.exp(-2.0 * 0.5 * 1.6), rel=0.01)


def test_sphere_normals_point_outward_and_face_the_camera_at_the_centre(cuda_device):
    _, image = render(sphere(grid16()))
    assert image[16, 16, NORMAL_Z] > 0.95
    assert image[16, 7, NORMAL_X] < -0.5  # the left edge faces left
    assert image[7, 16, NORMAL_Y] > 0.5  # the top edge faces up (row 0 is the top)


def test_empty_space_faces_the_camera(cuda_device):
    _, image = render(grid16())
    assert np.allclose(image[..., NORMAL_Z], 1.0) and np.all(image[..., THICKNESS] == 0.0)


def hot_cell_behind_a_smoke_wall():
    grid = grid16()
    temperature = np.full(CELLS, 293.0)
    temperature[7:9, 7:9, 2:4] = 1200.0  # far from the camera (low z)
    smoke = np.zeros(CELLS)
    smoke[:, :, 10:14] = 20.0  # a dense wall near the camera
    put(grid.temperature.data, temperature)
    put(grid.smoke.data, smoke)
    return grid


def test_smoke_in_front_hides_heat(cuda_device):
    _, hidden = render(hot_cell_behind_a_smoke_wall(), smoke_hides_heat=1.0)
    _, shown = render(hot_cell_behind_a_smoke_wall(), smoke_hides_heat=0.0)
    assert shown[16, 16, HEAT] > 10.0 and hidden[16, 16, HEAT] < 0.01 * shown[16, 16, HEAT]


def test_looking_straight_down_puts_the_back_at_the_top(cuda_device):
    grid = grid16()
    smoke = np.zeros(CELLS)
    smoke[6:10, 6:10, 1:4] = 2.0  # near the back face (low z)
    put(grid.smoke.data, smoke)
    view, image = render(grid, elevation_deg=90.0)
    rows = np.nonzero(image[..., THICKNESS].max(axis=1) > 0.1)[0]
    assert (view.width_px, view.height_px) == (32, 32) and rows.max() < 16


# ---- shading by the light volume (render/test_shade.py) ----------------------------------------------------

def shade_per_thickness(image):
    covered = image[..., THICKNESS] > 0.5
    return np.where(covered, image[..., SHADE] / np.maximum(image[..., THICKNESS], 0.5), np.nan)


def test_light_falls_through_a_uniform_slab_as_beer_lambert(cuda_device):
    from plume_b200.render.light_volume import LightVolume

    grid = grid16()
    grid.smoke.data.fill_(0.5)
    light = host(LightVolume(CELLS, np.array([0.0, 0.0, 1.0]), 2.0, "cuda:0").compute(grid.smoke.data, CELL_M))
    for k in (15, 8, 0):
        depth_m = (CELLS[2] - k - 0.5) * CELL_M  # from the cell centre to the +z face
        assert light[8, 8, k] == pytest.approx(math.exp(-2.0 * 0.5 * depth_m), rel=0.01), k


def test_a_sphere_lit_from_the_left_is_darker_on_its_right(cuda_device):
    _, image = render(sphere(grid16()), channels=SHADE_LAYOUT, light_dir=LEFT, shade_fill=0.25)
    shade = shade_per_thickness(image)
    assert np.nanmean(shade[:, :16]) > np.nanmean(shade[:, 16:]) + 0.2


def test_a_sphere_lit_from_above_is_darker_below(cuda_device):
    _, image = render(sphere(grid16()), elevation_deg=30.0, channels=SHADE_LAYOUT, light_dir=(0.0, 1.0, 0.0))
    shade = shade_per_thickness(image)
    assert np.nanmean(shade[:16]) > np.nanmean(shade[16:]) + 0.2


def test_light_from_the_camera_side_shows_more_than_light_from_behind(cuda_device):
    def mean_shade(light_dir):
        _, image = render(sphere(grid16()), elevation_deg=30.0, channels=SHADE_LAYOUT, light_dir=light_dir)
        covered = image[..., THICKNESS] > 0.5
        return float(np.mean(image[covered, SHADE] / image[covered, THICKNESS]))

    assert mean_shade((0.0, 0.0, 1.0)) > mean_shade((0.0, 0.0, -1.0)) + 0.2


def test_full_fill_casts_no_shadow(cuda_device):
    _, image = render(sphere(grid16()), channels=SHADE_LAYOUT, light_dir=LEFT, shade_fill=1.0)
    covered = image[..., THICKNESS] > 0.0
    assert np.allclose(image[covered, SHADE], image[covered, THICKNESS], atol=1e-5)
    shade = shade_per_thickness(image)
    assert np.nanmean(shade[:, :16]) == pytest.approx(np.nanmean(shade[:, 16:]), abs=1e-5)


def test_empty_space_has_no_shade(cuda_device):
    _, image = render(grid16(), channels=SHADE_LAYOUT)
    assert np.all(image[..., THICKNESS] == 0.0) and np.all(image[..., SHADE] == 0.0)


# ---- the perspective camera (render/test_view_cameras.py) --------------------------------------------------

def march(grid, renderer, params, height, width):
    import torch

    image = torch.zeros((height, width, CHANNELS), dtype=torch.float32, device="cuda:0")
    renderer.prepare(grid.smoke.data, grid.info.cell_m)
    renderer.march(grid.smoke.data, grid.temperature.data, grid.info, params, image)
    return host(image)


def test_a_far_narrow_perspective_camera_matches_the_orthographic_march(cuda_device):
    from plume_b200.render.frame_renderer import FrameRenderer, domain_view_params

    grid = grid16()
    put(grid.smoke.data, 3.0 * blob(CELLS, (8.0, 7.0, 9.0), 3.0))
    put(grid.temperature.data, 293.0 + 900.0 * blob(CELLS, (8.0, 7.0, 9.0), 2.0))
    view = box_view(25.0, 40.0)
    renderer = FrameRenderer(view, RenderSettings(), grid.cells, SHADE_LAYOUT, "cuda:0")
    orthographic = march(grid, renderer, renderer.view_params, view.height_px, view.width_px)
    # an eye 200 m out along the view axis, its image plane at the origin scaled to the domain view's pixels
    distance = 200.0
    cx = view.left_m + view.width_px * view.pixel_m / 2
    cy = view.top_m - view.height_px * view.pixel_m / 2
    params = domain_view_params(view)
    params.perspective = 1
    params.eye = type(params.eye)(*(view.camera.right * cx + view.camera.up * cy + view.camera.toward * distance))
    params.left_m, params.top_m = (view.left_m - cx) / distance, (view.top_m - cy) / distance
    params.pixel_m = view.pixel_m / distance
    perspective = march(grid, renderer, params, view.height_px, view.width_px)
    assert np.abs(perspective[..., THICKNESS] - orthographic[..., THICKNESS]).max() < 0.01
    assert np.abs(perspective[..., SHADE] - orthographic[..., SHADE]).max() < 0.01
    assert np.abs(perspective[..., HEAT] - orthographic[..., HEAT]).max() < 0.01 * orthographic[..., HEAT].max()
    assert orthographic[..., THICKNESS].max() > 0.9


def test_an_eye_inside_the_smoke_sees_only_what_is_in_front(cuda_device):
    from plume_b200.render.frame_renderer import FrameRenderer, domain_view_params

    grid = grid16()
    grid.smoke.data.fill_(0.5)
    view = box_view()
    renderer = FrameRenderer(view, RenderSettings(opacity_per_density=2.0), grid.cells, SHADE_LAYOUT, "cuda:0")
    params = domain_view_params(view)
    params.perspective = 1
    params.eye = type(params.eye)(0.0, 0.8, 0.3)  # 1.1 m from the back wall (z = -0.8), looking along -z
    params.left_m, params.top_m, params.pixel_m = -0.5, 0.5, 1.0 / 9.0
    image = march(grid, renderer, params, 9, 9)
    assert image[4, 4, THICKNESS] == pytest.approx(1.0 - math.exp(-2.0 * 0.5 * 1.1), rel=1e-4)
