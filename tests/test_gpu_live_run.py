"""The viewer's headless run (tests/view/test_live_run.py and test_frame_cache.py in chadmv/plume): the live
run's frames are `plume run`'s raw frames byte for byte, its cache holds the run's fields rounded to 16 bits,
its divisors are the sheet's, and the frame cache keeps, thins and widens frames as planned."""

import numpy as np
import pytest

from support import host, put, tiny_recipe

pytestmark = pytest.mark.gpu

HOT = [{"name": "puff", "center_m": [0.0, 0.3, 0.0], "radius_m": 0.2, "end_s": 0.5, "smoke_per_s": 5.0,
        "temperature_k": 900.0}]
CELLS = (8, 6, 4)


def run_like_plume_run(recipe, derived):
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.run import simulate

    view = sheet_domain_view(recipe, derived)
    renderer = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "cuda:0")
    raw_frames, smokes = [], []

    def capture(frame, grid):
        raw_frames.append(renderer.render(grid))
        smokes.append(host(grid.smoke.data).copy())

    simulate(recipe, derived, "cuda:0", capture)
    return raw_frames, smokes, view


@pytest.fixture(scope="module")
def runs(cuda_device):
    from plume_b200.recipe.derived import derive
    from plume_b200.view.live_run import LiveRun

    recipe = tiny_recipe(emitter=HOT, camera={"elevation_deg": 15.0})
    derived = derive(recipe)
    live = LiveRun(recipe, derived, "cuda:0", budget_bytes=1e9)
    while live.advance() is not None:
        pass
    live.wait_for_assembly()
    return recipe, derived, live, run_like_plume_run(recipe, derived)


def test_every_frame_is_plume_runs_raw_frame_byte_for_byte(runs):
    _, _, live, (raw_frames, _, _) = runs
    assert live.done and live.landed == len(raw_frames) == 4
    for viewer_frame, run_frame in zip(live.raw_frames, raw_frames, strict=True):
        assert viewer_frame.tobytes() == run_frame.tobytes()


def test_every_kept_smoke_is_the_runs_smoke_rounded_to_16_bits(runs):
    _, _, live, (_, smokes, _) = runs
    assert live.cache.kept_frames() == [0, 1, 2, 3]
    for frame, smoke in enumerate(smokes):
        assert np.array_equal(host(live.cache.stored_smoke(frame)), smoke.astype(np.float16))


def test_the_divisors_are_the_sheets(runs):
    from plume_b200.run import seat_point
    from plume_b200.sheet.assemble import assemble

    recipe, _, live, (raw_frames, _, view) = runs
    sheet = assemble(raw_frames, view, seat_point(recipe), recipe.output.frame_px, recipe.render,
                     recipe.output.channels)
    assert live.assembled is not None and live.assembly_error is None
    assert live.heat_divisor == sheet.heat_divisor > 0.0 and live.shade_divisor == sheet.shade_divisor
    assert live.assembled.crop == sheet.crop
    assert live.steps.total_steps > 0 and live.elapsed_s > 0.0


def test_a_run_keeps_velocity_and_notes_edges_every_frame(runs):
    _, _, live, _ = runs
    assert live.cache.has_velocity and all(live.cache.velocity_kept(frame) for frame in range(4))
    assert sorted(live.edges) == [0, 1, 2, 3]


def test_a_recapture_renders_the_kept_frames_again(runs):
    import dataclasses

    from plume_b200.view.live_run import LiveRun

    recipe, _, live, _ = runs
    edited = dataclasses.replace(recipe, render=dataclasses.replace(recipe.render, opacity_per_density=2.0 *
                                                                    recipe.render.opacity_per_density))
    again = LiveRun.recapture(live, edited)
    assert again.heat_divisor == live.heat_divisor  # the source's until its own assembly lands
    while again.advance() is not None:
        pass
    assert again.landed == 4 and again.assembled is not None
    assert again.raw_frames[-1][..., 1].max() > live.raw_frames[-1][..., 1].max()  # denser smoke


def test_before_assembly_heat_uses_the_largest_raw_heat_so_far(cuda_device):
    from plume_b200.recipe.derived import derive
    from plume_b200.view.live_run import LiveRun

    recipe = tiny_recipe(emitter=HOT)
    live = LiveRun(recipe, derive(recipe), "cuda:0", budget_bytes=1e9)
    live.advance()
    live.advance()
    assert live.heat_divisor == max(float(frame[..., 0].max()) for frame in live.raw_frames)
    assert live.shade_divisor == 1.0
    live.cancel()
    assert not live.done and live.stopped and live.advance() is None


def test_the_boundary_layers_are_the_smokes_outer_cells(cuda_device):
    import torch

    from plume_b200.view.live_run import boundary_layers

    smoke = np.arange(3 * 4 * 5, dtype=np.float32).reshape(3, 4, 5)
    got = host(boundary_layers(torch.from_numpy(smoke).cuda()))
    assert np.array_equal(got[0, :4, :5], smoke[0]) and np.array_equal(got[1, :4, :5], smoke[-1])
    assert np.array_equal(got[2, :3, :5], smoke[:, 0]) and np.array_equal(got[3, :3, :5], smoke[:, -1])
    assert np.array_equal(got[4, :3, :4], smoke[:, :, 0]) and np.array_equal(got[5, :3, :4], smoke[:, :, -1])
    assert got[0, 4].sum() == 0.0 and got[2, 3].sum() == 0.0


# ---- the frame cache (view/test_frame_cache.py) --------------------------------------------------------------

def device(values):
    import torch

    return torch.from_numpy(np.asarray(values, dtype=np.float32)).cuda()


def test_a_stored_frame_is_the_field_rounded_to_16_bits(cuda_device):
    from plume_b200.view.frame_cache import FrameCache

    rng = np.random.default_rng(5)
    smoke = rng.uniform(0.0, 3.0, CELLS).astype(np.float32)
    temperature = rng.uniform(290.0, 1500.0, CELLS).astype(np.float32)
    cache = FrameCache(CELLS, frames=4, budget_bytes=1e9, device="cuda:0")
    cache.store(0, device(smoke), device(temperature))
    assert np.array_equal(host(cache.stored_smoke(0)), smoke.astype(np.float16))
    wide_smoke, wide_temperature = cache.load(0, cache.scratch())
    assert np.array_equal(host(wide_smoke), smoke.astype(np.float16).astype(np.float32))
    assert np.array_equal(host(wide_temperature), temperature.astype(np.float16).astype(np.float32))


def test_a_kept_velocity_is_the_centred_velocity_rounded_to_16_bits(cuda_device):
    from plume_b200.view.frame_cache import FrameCache, frame_bytes

    rng = np.random.default_rng(7)
    nx, ny, nz = CELLS
    u = rng.uniform(-2.0, 2.0, (nx + 1, ny, nz)).astype(np.float32)
    v = rng.uniform(-2.0, 2.0, (nx, ny + 1, nz)).astype(np.float32)
    w = rng.uniform(-2.0, 2.0, (nx, ny, nz + 1)).astype(np.float32)
    zeros = device(np.zeros(CELLS))
    cache = FrameCache(CELLS, frames=2, budget_bytes=1e9, device="cuda:0")
    cache.store(0, zeros, zeros, (device(u), device(v), device(w)))
    centred = np.stack([0.5 * (u[:-1] + u[1:]), 0.5 * (v[:, :-1] + v[:, 1:]), 0.5 * (w[:, :, :-1] + w[:, :, 1:])],
                       axis=-1).astype(np.float32)
    assert cache.velocity_kept(0)
    assert np.array_equal(host(cache.load_velocity(0, cache.velocity_scratch())),
                          centred.astype(np.float16).astype(np.float32))
    assert cache.stored_bytes == frame_bytes(CELLS, velocity=True)


def test_a_thinned_cache_skips_frames_and_says_so(cuda_device):
    from plume_b200.view.frame_cache import FrameCache, frame_bytes

    cache = FrameCache(CELLS, frames=8, budget_bytes=4 * frame_bytes(CELLS), device="cuda:0")
    zeros = device(np.zeros(CELLS))
    for frame in range(8):
        cache.store(frame, zeros, zeros)
    assert cache.kept_frames() == [0, 2, 4, 6] and cache.nearest_kept(5) == 4 and not cache.has_velocity
    assert "every 2nd frame and no velocity" in cache.thinning_note()
    assert FrameCache(CELLS, frames=8, budget_bytes=1e9, device="cuda:0").thinning_note() is None
