"""Render parity: light volume, normal field and ray march (both layouts, orthographic and perspective)
through the C ABI against the FP32 oracle. exp/pow are evaluated in double on the device and as expf/powf in
the oracle, so values agree to about an ulp per call; the march accumulates them (tolerance below)."""

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.schema import NORMAL_LAYOUT, SHADE_LAYOUT, RenderSettings
from plume_b200.render.camera import make_camera, make_domain_view
from plume_b200.workloads import operator_fields
from support import OPEN, assert_same, blob, cuda_grid, host, load_state, max_rel, oracle_grid

pytestmark = pytest.mark.gpu

LIGHT_RTOL = 1e-5
MARCH_ATOL = 1e-5


def render_pair(cells=(24, 32, 20), seed=4):
    o = oracle_grid(cells, 0.05, OPEN, 293.0)
    c = cuda_grid(cells, 0.05, OPEN, 293.0)
    fields = operator_fields(cells, seed, 293.0)
    fields["temperature"] = (293.0 + 900.0 * blob(cells, [n / 2 for n in cells], 3.0)).astype(np.float32)
    fields["smoke"] = (3.0 * fields["smoke"]).astype(np.float32)
    load_state(o, c, fields)
    return o, c


def test_light_volume_matches_the_oracle(cuda_device):
    from plume_b200.render.light_volume import LightVolume

    o, c = render_pair()
    direction = np.array([0.5, 0.8, 0.3])
    light = LightVolume(c.cells, direction, 4.0, "cuda:0").compute(c.smoke.data, c.info.cell_m)
    expected = O.light_volume(o.smoke.data, direction, o.cell_m, 4.0)
    assert max_rel(host(light), expected, floor=1e-6) < LIGHT_RTOL


@pytest.mark.parametrize("cells", [(24, 32, 20), (64, 96, 64)])
def test_light_volume_empty_space_skipping_changes_no_bit(cuda_device, cells):
    """The brick map only steps over samples that add exactly 0: the light volume is bit-identical without it."""
    import torch

    from plume_b200 import _native as N

    o, c = render_pair(cells)
    smoke = c.smoke.data
    toward = N.f3(np.array([0.5, 0.8, 0.3]) / np.linalg.norm([0.5, 0.8, 0.3]))
    with_bricks, without = torch.empty_like(smoke), torch.empty_like(smoke)
    bricks = torch.empty(N.lib().plume_brick_floats(N.shape3(smoke)), dtype=torch.float32, device="cuda:0")
    N.call("plume_light_volume", N.shape3(smoke), N.ptr(smoke), 0, toward, 0.05, 4.0, N.ptr(with_bricks),
           N.ptr(bricks), N.stream())
    N.call("plume_light_volume", N.shape3(smoke), N.ptr(smoke), 0, toward, 0.05, 4.0, N.ptr(without), None, N.stream())
    assert torch.equal(with_bricks, without)
    assert float((smoke <= 0).float().mean()) > 0.5  # the case has plenty of empty space to skip


@pytest.mark.parametrize("channels", [SHADE_LAYOUT, NORMAL_LAYOUT])
@pytest.mark.parametrize("elevation,azimuth", [(0.0, 0.0), (20.0, 30.0), (90.0, 0.0), (-35.0, 200.0)])
def test_frame_matches_the_oracle(cuda_device, channels, elevation, azimuth):
    from plume_b200.render.frame_renderer import FrameRenderer

    o, c = render_pair()
    cells = c.cells
    size = tuple(n * 0.05 for n in cells)
    view = make_domain_view(make_camera(elevation, azimuth), (-size[0] / 2, 0.0, -size[2] / 2), size, 0.05, 2.0)
    settings = RenderSettings(glow_start_k=600.0, light_dir=(0.5, 0.8, 0.3))
    image = FrameRenderer(view, settings, cells, channels, "cuda:0").render(c)
    expected = O.FrameRenderer(view, settings, cells, channels).render(o)
    assert image.shape == expected.shape == (view.height_px, view.width_px, 5)
    heat_scale = max(float(np.abs(expected[..., 0]).max()), 1.0)
    assert np.abs(image[..., 0] - expected[..., 0]).max() < MARCH_ATOL * heat_scale * 10
    assert np.abs(image[..., 1:] - expected[..., 1:]).max() < MARCH_ATOL * 10


@pytest.mark.parametrize("channels", [SHADE_LAYOUT, NORMAL_LAYOUT])
@pytest.mark.parametrize("glow_start", [600.0, 293.0])  # 293 K is the ambient: one-valued bricks cannot glow
@pytest.mark.parametrize("cells,perspective", [((24, 32, 20), False), ((64, 96, 64), False), ((64, 96, 64), True)])
def test_march_empty_space_skipping_changes_no_bit(cuda_device, channels, glow_start, cells, perspective):
    """The march's brick map only skips samples and runs of samples that add exactly 0: the image is
    bit-identical without it, orthographic (origin 1e4 m out, the largest rounding of the sample points) and
    perspective."""
    import torch

    from plume_b200 import _native as N
    from plume_b200.render.frame_renderer import FrameRenderer

    o, c = render_pair(cells)
    size = tuple(n * 0.05 for n in cells)
    view = make_domain_view(make_camera(20.0, 30.0), (-size[0] / 2, 0.0, -size[2] / 2), size, 0.05, 2.0)
    renderer = FrameRenderer(view, RenderSettings(glow_start_k=glow_start, light_dir=(0.5, 0.8, 0.3)), cells,
                             channels, "cuda:0")
    params = renderer.view_params
    if perspective:  # an eye 3 m out along the view axis from the box centre
        centre = np.array([c.info.origin_m[a] + 0.5 * cells[a] * 0.05 for a in range(3)])
        params.perspective = 1
        params.eye = type(params.eye)(*(centre + 3.0 * view.camera.toward))
        params.left_m, params.top_m = -0.5 * renderer.image.shape[1] / 256, 0.5 * renderer.image.shape[0] / 256
        params.pixel_m = 1.0 / 256
    renderer.prepare(c.smoke.data, c.info.cell_m)
    skipped = torch.zeros_like(renderer.image)
    full = torch.zeros_like(renderer.image)
    renderer.march(c.smoke.data, c.temperature.data, c.info, params, skipped)
    N.call("plume_raymarch", c.info, N.ptr(c.smoke.data), N.ptr(c.temperature.data), 0, N.ptr(renderer.gradient),
           N.c_int3(*renderer.gradient.shape[:3]), N.ptr(renderer.light), N.shape3(renderer.light),
           params, renderer.look_params, N.ptr(full), full.shape[0], full.shape[1], None, N.stream())
    assert torch.equal(skipped, full)
    assert float(full[..., 1].max()) > 0.1  # the rays cross smoke
    if glow_start < 300.0:
        assert float(full[..., 0].max()) > 0.0  # and glow


def read_by_march(smoke: np.ndarray) -> np.ndarray:
    """Cells whose light a march of `smoke` can read: one of the 27 cells around it holds smoke > 0 (a sample
    reads the light at its corners only when one of them holds smoke > 0)."""
    n = smoke.shape
    padded = np.pad(smoke > 0, 1)
    read = np.zeros(n, dtype=bool)
    for a in range(3):
        for b in range(3):
            for c in range(3):
                read |= padded[a:a + n[0], b:b + n[1], c:c + n[2]]
    return read


@pytest.mark.parametrize("cells", [(24, 32, 20), (64, 96, 64)])
def test_march_light_volume_is_the_light_volume_where_the_march_reads(cuda_device, cells):
    """plume_march_light_volume: the read cells bit for bit as plume_light_volume, 1 elsewhere; and the frame a
    renderer marches with it is bit-identical to one marched with the whole light volume."""
    import torch

    from plume_b200 import _native as N
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.render.light_volume import LightVolume

    o, c = render_pair(cells)
    direction = np.array([0.5, 0.8, 0.3])
    whole = LightVolume(c.cells, direction, 4.0, "cuda:0").compute(c.smoke.data, c.info.cell_m).clone()
    marched = LightVolume(c.cells, direction, 4.0, "cuda:0").compute(c.smoke.data, c.info.cell_m, march_cells=True)
    read = read_by_march(host(c.smoke.data))
    assert 0.05 < read.mean() < 0.9
    assert np.array_equal(host(marched)[read], host(whole)[read])
    assert np.all(host(marched)[~read] == 1.0)

    size = tuple(n * 0.05 for n in cells)
    view = make_domain_view(make_camera(20.0, 30.0), (-size[0] / 2, 0.0, -size[2] / 2), size, 0.05, 2.0)
    renderer = FrameRenderer(view, RenderSettings(glow_start_k=600.0, light_dir=tuple(direction)), cells,
                             SHADE_LAYOUT, "cuda:0")
    image = renderer.render(c)
    renderer.light = renderer.light_volume.compute(c.smoke.data, c.info.cell_m).clone()  # the whole light volume
    renderer.march(c.smoke.data, c.temperature.data, c.info, renderer.view_params, renderer.image)
    assert np.array_equal(image, host(renderer.image))


def test_normal_field_matches_the_oracle(cuda_device):
    from plume_b200.render.normal_field import NormalField

    o, c = render_pair()
    field = NormalField(c.cells, 1.5, "cuda:0")
    gradient = field.compute(c.smoke.data)
    renderer = O.FrameRenderer(make_domain_view(make_camera(0, 0), (0, 0, 0), (1, 1, 1), 0.05, 2.0),
                               RenderSettings(), c.cells, NORMAL_LAYOUT)
    renderer.prepare(o.smoke.data, o.cell_m)
    assert_same(host(gradient), renderer.gradient, "gradient")


def test_perspective_march_matches_the_oracle(cuda_device):
    import torch

    from plume_b200.render.frame_renderer import FrameRenderer, domain_view_params

    o, c = render_pair()
    cells = c.cells
    size = tuple(n * 0.05 for n in cells)
    view = make_domain_view(make_camera(25.0, 40.0), (-size[0] / 2, 0.0, -size[2] / 2), size, 0.05, 2.0)
    settings = RenderSettings()
    renderer = FrameRenderer(view, settings, cells, SHADE_LAYOUT, "cuda:0")
    oracle = O.FrameRenderer(view, settings, cells, SHADE_LAYOUT)
    params = domain_view_params(view)
    params.perspective = 1
    params.eye = type(params.eye)(0.1, 0.6, 0.2)  # inside the domain
    params.left_m, params.top_m, params.pixel_m = -0.5, 0.5, 1.0 / 9.0
    image = torch.zeros((9, 9, 5), dtype=torch.float32, device="cuda:0")
    renderer.prepare(c.smoke.data, c.info.cell_m)
    renderer.march(c.smoke.data, c.temperature.data, c.info, params, image)
    oparams = O.domain_view_params(view)
    oparams.perspective = 1
    oparams.eye = O._d3((0.1, 0.6, 0.2))
    oparams.left_m, oparams.top_m, oparams.pixel_m = -0.5, 0.5, 1.0 / 9.0
    expected = np.zeros((9, 9, 5), dtype=np.float32)
    oracle.prepare(o.smoke.data, o.cell_m)
    oracle.march(o.smoke.data, o.temperature.data, o.info, oparams, expected)
    assert np.abs(host(image)[..., 1:] - expected[..., 1:]).max() < MARCH_ATOL * 10


@pytest.mark.parametrize("channels", [SHADE_LAYOUT, NORMAL_LAYOUT])
def test_render_async_gives_the_frames_render_gives(cuda_device, channels):
    """Frames enqueued by render_async while the next substeps already run are bit-identical to render()."""
    import torch

    from plume_b200.recipe.derived import derive
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper
    from plume_b200.workloads import operator_fields, plain_step_recipe

    recipe = plain_step_recipe((32, 48, 32), cycles=2)
    derived = derive(recipe)
    d = recipe.domain
    frames = {}
    for arm in ("sync", "async"):
        grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0")
        for name, values in operator_fields(derived.cells, 5, d.ambient_k).items():
            getattr(grid, name).data.copy_(torch.from_numpy(values))
        stepper = Stepper(grid, recipe)
        renderer = FrameRenderer(sheet_domain_view(recipe, derived), recipe.render, derived.cells, channels, "cuda:0")
        out = []
        for frame in range(4):
            for n in range(2):
                stepper.step((2 * frame + n) * derived.dt_s, derived.dt_s)
            out.append(renderer.render(grid) if arm == "sync" else renderer.render_async(grid))
        frames[arm] = out if arm == "sync" else [pending.result() for pending in out]
    for index, (a, b) in enumerate(zip(frames["sync"], frames["async"])):
        assert np.array_equal(a, b), f"frame {index}"
    assert frames["sync"][-1][..., 1].max() > 0.1


def test_bfloat16_storage_skips_and_lights_exactly_as_without_the_shortcuts(cuda_device):
    """With bfloat16 fields: the light volume a march reads equals the whole light volume at the read cells,
    and the march with its brick map equals the march without it, bit for bit."""
    import torch

    from plume_b200 import _native as N
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from support import small_derived

    cells = (48, 64, 40)
    _, c = render_pair(cells)
    g = make_grid(small_derived(cells, 0.05), 0.05, OPEN, 293.0, "cuda:0", storage=torch.bfloat16)
    for name in ("u", "v", "w", "smoke", "temperature"):
        getattr(g, name).data.copy_(getattr(c, name).data)
    smoke = g.smoke.data
    toward = N.f3(np.array([0.5, 0.8, 0.3]) / np.linalg.norm([0.5, 0.8, 0.3]))
    bricks = torch.empty(N.lib().plume_brick_floats(N.shape3(smoke)), dtype=torch.float32, device="cuda:0")
    whole = torch.empty(cells, dtype=torch.float32, device="cuda:0")
    marched = torch.empty_like(whole)
    N.call("plume_light_volume", N.shape3(smoke), N.field_ptr(smoke), N.storage_of(smoke), toward, 0.05, 4.0,
           N.ptr(whole), N.ptr(bricks), N.stream())
    N.call("plume_march_light_volume", N.shape3(smoke), N.field_ptr(smoke), N.storage_of(smoke), toward, 0.05, 4.0,
           N.ptr(marched), N.ptr(bricks), N.stream())
    read = read_by_march(host(smoke.float()))
    assert np.array_equal(host(marched)[read], host(whole)[read]) and np.all(host(marched)[~read] == 1.0)

    size = tuple(n * 0.05 for n in cells)
    view = make_domain_view(make_camera(20.0, 30.0), (-size[0] / 2, 0.0, -size[2] / 2), size, 0.05, 2.0)
    renderer = FrameRenderer(view, RenderSettings(glow_start_k=293.0, light_dir=(0.5, 0.8, 0.3)), cells,
                             SHADE_LAYOUT, "cuda:0")
    renderer.prepare(smoke, g.info.cell_m)
    skipped, full = torch.zeros_like(renderer.image), torch.zeros_like(renderer.image)
    renderer.march(smoke, g.temperature.data, g.info, renderer.view_params, skipped)
    N.call("plume_raymarch", g.info, N.field_ptr(smoke), N.field_ptr(g.temperature.data), N.storage_of(smoke),
           N.ptr(renderer.gradient), N.c_int3(*renderer.gradient.shape[:3]), N.ptr(renderer.light),
           N.shape3(renderer.light), renderer.view_params, renderer.look_params, N.ptr(full), full.shape[0],
           full.shape[1], None, N.stream())
    assert torch.equal(skipped, full) and float(full[..., 1].max()) > 0.1
