"""The viewer's device compute against the viewer oracle: the look bytes exactly (and within a byte of the
host composite), the centre ray's depth to within one march step, the centre velocity, curl, speed, slice
overlay and boundary layers exactly, the float16 casts as torch's."""

import numpy as np
import pytest

from oracle import view as V
from plume_b200.recipe.schema import LookSettings
from plume_b200.view.color import hex_to_linear, ramp, to_srgb_bytes
from support import ALL_CLOSED, OPEN, blob, cuda_grid, host
from test_view_oracle import BACKGROUND, HEAT_DIVISOR, LIGHT_DIR, SHADE_DIVISOR, byte_grid, raw_from_pixels

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shade", [True, False])
@pytest.mark.parametrize("view", [0, 1, 2, 3])
def test_look_bytes_match_the_oracle(cuda_device, shade, view):
    from types import SimpleNamespace

    from plume_b200.view.viewport import LookTables, look_bytes, look_inputs

    channels = "heat,thickness,shade,unused" if shade else "heat,thickness,normal_x,normal_y"
    recipe = SimpleNamespace(look=LookSettings(), output=SimpleNamespace(channels=channels))
    rgba = byte_grid(shade)
    raw = raw_from_pixels(rgba, shade)
    toward = np.array(LIGHT_DIR) / np.linalg.norm(LIGHT_DIR)
    tables = LookTables(recipe, "cuda:0")
    got = look_bytes(raw, tables, look_inputs(recipe, view, HEAT_DIVISOR, SHADE_DIVISOR, BACKGROUND, toward), "cuda:0")
    f32 = lambda x: np.float32(x)  # noqa: E731  (the kernel's inputs are float32)
    want = V.look(raw, host(tables.smoke_ramp), host(tables.emission_ramp), host(tables.srgb), view, shade,
                  f32(HEAT_DIVISOR), f32(SHADE_DIVISOR), f32(0.75), f32(0.65), toward.astype(np.float32),
                  hex_to_linear(BACKGROUND).astype(np.float32))
    assert np.array_equal(got, want)
    if view == 0:
        look = LookSettings()
        expected = to_srgb_bytes(V.composite(rgba, hex_to_linear(BACKGROUND), shade, look, LIGHT_DIR, ramp))
        assert np.abs(got[..., :3].astype(int) - expected.astype(int)).max() <= 1


def puff_grid(faces=OPEN):
    import torch

    cells = (20, 28, 16)
    c = cuda_grid(cells, 0.05, faces)
    smoke = (2.0 * blob(cells, (10, 9, 8), 3.5)).astype(np.float32)
    c.smoke.data.copy_(torch.from_numpy(smoke))
    rng = np.random.default_rng(4)
    for f in c.velocity_fields():
        f.data.copy_(torch.from_numpy(rng.uniform(-1, 1, tuple(f.data.shape)).astype(np.float32)))
    return c, smoke


def test_center_depth_matches_the_oracle(cuda_device):
    from plume_b200.view.viewport import center_depth

    c, smoke = puff_grid()
    origin_m = tuple(c.info.origin_m)
    for origin, direction in (((0.0, 0.45, 3.0), (0.0, 0.0, -1.0)), ((-2.0, 0.9, -1.0), (0.8, -0.2, 0.3)),
                              ((0.0, 0.45, 3.0), (0.0, 0.0, 1.0))):
        direction = np.array(direction) / np.linalg.norm(direction)
        got = center_depth(c.smoke.data, c.info, origin, direction, 4.0, 0.5)
        want = V.center_depth(smoke, origin_m, 0.05, origin, direction, 4.0, 0.5)
        assert (got < 0) == (want < 0)
        assert abs(got - want) <= 0.5 * 0.05 + 1e-6  # at most one half-cell step apart


def test_slice_fields_and_overlay_match_the_oracle(cuda_device):
    import torch

    from plume_b200.render.camera import make_camera, make_domain_view
    from plume_b200.render.frame_renderer import domain_view_params
    from plume_b200.view.slice_plane import SliceDrawer, center_velocity, curl, speed

    c, smoke = puff_grid()
    u, v, w = (host(f.data) for f in c.velocity_fields())
    centers = center_velocity(c)
    assert np.array_equal(host(centers), V.center_velocity(u, v, w))
    swirl = curl(c.info, centers)
    assert np.array_equal(host(swirl), V.curl(host(centers), 0.05))
    values = speed(swirl)
    assert np.array_equal(host(values), V.speed(host(swirl)))
    size = tuple(n * 0.05 for n in c.cells)
    view = domain_view_params(make_domain_view(make_camera(20.0, 30.0), tuple(c.info.origin_m), size, 0.05, 1.0))
    image = torch.from_numpy(np.random.default_rng(1).integers(0, 256, (24, 30, 4), dtype=np.uint8)).cuda()
    before = host(image)
    low, high = 0.0, float(values.max())
    for axis, coordinate in ((0, -0.1), (1, 0.7), (2, 0.0)):
        drawn = image.clone()
        SliceDrawer("cuda:0").overlay(drawn, view, c.info, axis, coordinate, values, low, high)
        want = V.slice_overlay(view, tuple(c.info.origin_m), 0.05, axis, coordinate, host(values), low, high,
                               host(SliceDrawer("cuda:0").ramp), before)
        assert np.array_equal(host(drawn), want), axis


def test_boundary_layers_and_float16_casts(cuda_device):
    import torch

    from plume_b200.view.live_run import boundary_layers, narrow, widen

    c, smoke = puff_grid(ALL_CLOSED)
    assert np.array_equal(host(boundary_layers(c.smoke.data)), V.boundary_layers(smoke))
    half = narrow(c.smoke.data)
    assert torch.equal(half, c.smoke.data.half())
    assert torch.equal(widen(half), half.float())
