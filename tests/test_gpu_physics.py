"""The reference's physics-property tests of the simulation (tests/sim/*.py in chadmv/plume), run on the CUDA
path: each states a property of the method (a blob carried by a uniform flow, divergence removed, a vortex
spun up, an emitter's output, the CFL cap, conservation) with the reference's bounds."""

import math

import numpy as np
import pytest

from support import ALL_CLOSED, OPEN, blob, cuda_grid, host, put, tiny_recipe

pytestmark = pytest.mark.gpu


def velocity(grid):
    return tuple(f.data for f in grid.velocity_fields())


# ---- advection (sim/test_advect.py) -----------------------------------------------------------------------

def swirl(grid):
    """A closed 2-D circulation in x-y: u = sin(pi x) cos(pi y), v = -cos(pi x) sin(pi y) at the faces."""
    nx, ny, nz = grid.cells
    x = np.arange(nx + 1)[:, None, None] / nx
    y = (np.arange(ny)[None, :, None] + 0.5) / ny
    put(grid.u.data, np.broadcast_to(np.sin(np.pi * x) * np.cos(np.pi * y), (nx + 1, ny, nz)))
    x = (np.arange(nx)[:, None, None] + 0.5) / nx
    y = np.arange(ny + 1)[None, :, None] / ny
    put(grid.v.data, np.broadcast_to(-np.cos(np.pi * x) * np.sin(np.pi * y), (nx, ny + 1, nz)))


def mass_centre_x(values):
    weights = values.sum(axis=(1, 2))
    return float((weights * (np.arange(values.shape[0]) + 0.5)).sum() / weights.sum())


def test_a_constant_field_stays_constant(cuda_device):
    from plume_b200.sim.advect import advect_maccormack

    grid = cuda_grid()
    swirl(grid)
    grid.smoke.data.fill_(1.0)
    for _ in range(5):
        advect_maccormack(grid.smoke, velocity(grid), grid, 0.05)
        grid.smoke.swap()
    assert np.abs(host(grid.smoke.data) - 1.0).max() <= 1e-5


def test_a_blob_travels_with_a_uniform_flow(cuda_device):
    from plume_b200.sim.advect import advect_maccormack

    grid = cuda_grid(cells=(32, 12, 12))
    grid.u.data.fill_(1.0)  # 10 cells per second
    put(grid.smoke.data, blob(grid.cells, (8.0, 6.0, 6.0), 2.0))
    start = mass_centre_x(host(grid.smoke.data))
    for _ in range(20):
        advect_maccormack(grid.smoke, velocity(grid), grid, 0.05)
        grid.smoke.swap()
    assert mass_centre_x(host(grid.smoke.data)) - start == pytest.approx(10.0, abs=0.5)


def test_maccormack_keeps_a_peak_sharper_than_semi_lagrangian(cuda_device):
    from plume_b200.sim.advect import advect_maccormack, advect_semi_lagrangian

    peaks = {}
    for name, advect in (("semi_lagrangian", advect_semi_lagrangian), ("maccormack", advect_maccormack)):
        grid = cuda_grid(cells=(32, 12, 12))
        grid.u.data.fill_(0.37)
        put(grid.smoke.data, blob(grid.cells, (8.0, 6.0, 6.0), 1.5))
        for _ in range(20):
            advect(grid.smoke, velocity(grid), grid, 0.05)
            grid.smoke.swap()
        peaks[name] = float(grid.smoke.data.max())
    assert peaks["maccormack"] > 1.1 * peaks["semi_lagrangian"]


def test_the_clamp_makes_no_new_extremes(cuda_device):
    from plume_b200.sim.advect import advect_maccormack

    grid = cuda_grid()
    swirl(grid)
    start = np.random.default_rng(3).random(grid.cells)
    put(grid.smoke.data, start)
    advect_maccormack(grid.smoke, velocity(grid), grid, 0.1)
    grid.smoke.swap()
    result = host(grid.smoke.data)
    assert result.min() >= start.min() - 1e-6 and result.max() <= start.max() + 1e-6


# ---- projection and multigrid (sim/test_pressure.py, sim/test_multigrid.py) -------------------------------

def random_velocity(grid, seed=5):
    rng = np.random.default_rng(seed)
    for field in grid.velocity_fields():
        put(field.data, rng.normal(size=tuple(field.data.shape)))


def divergence_norm(grid):
    from plume_b200.sim.pressure import compute_divergence

    return float(np.linalg.norm(host(compute_divergence(grid))))


@pytest.mark.parametrize("faces", [ALL_CLOSED, OPEN], ids=["closed", "open"])
def test_sixty_gauss_seidel_sweeps_remove_most_divergence(cuda_device, faces):
    from plume_b200.sim.pressure import GaussSeidel, project

    grid = cuda_grid(faces=faces)
    random_velocity(grid)
    project(grid, GaussSeidel(0))  # closes the walls; nothing solved yet
    before = divergence_norm(grid)
    project(grid, GaussSeidel(60))
    assert divergence_norm(grid) < 0.1 * before


def test_a_closed_floor_has_no_normal_velocity_and_an_open_top_has_some(cuda_device):
    from plume_b200.sim.pressure import GaussSeidel, project

    grid = cuda_grid(faces=OPEN)
    random_velocity(grid)
    project(grid, GaussSeidel(20))
    v = host(grid.v.data)
    assert np.all(v[:, 0, :] == 0.0) and np.any(v[:, -1, :] != 0.0)


def jet(cells, faces):
    """A smooth upward jet: a Gaussian blob of v, radius a fifth of the shortest axis."""
    grid = cuda_grid(cells=cells, faces=faces)
    shape = tuple(grid.v.data.shape)
    put(grid.v.data, blob(shape, [n / 2 for n in shape], min(cells) / 5))
    return grid


def divergence_left(grid, solve):
    from plume_b200.sim.pressure import GaussSeidel, project

    project(grid, GaussSeidel(0))
    before = divergence_norm(grid)
    project(grid, solve)
    return divergence_norm(grid) / before


@pytest.mark.parametrize("faces", [ALL_CLOSED, OPEN], ids=["closed", "open"])
@pytest.mark.parametrize("cells", [(32, 32, 32), (31, 33, 29)], ids=["even", "odd"])
def test_two_v_cycles_beat_sixty_gauss_seidel_sweeps(cuda_device, cells, faces):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import GaussSeidel

    grid = jet(cells, faces)
    multigrid = divergence_left(grid, Multigrid(grid, 2, 2))
    gauss_seidel = divergence_left(jet(cells, faces), GaussSeidel(60))
    assert multigrid < 0.1 and multigrid < 0.25 * gauss_seidel


@pytest.mark.parametrize("faces", [ALL_CLOSED, OPEN], ids=["closed", "open"])
def test_each_v_cycle_at_least_halves_the_residual(cuda_device, faces):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import GaussSeidel, compute_divergence, project

    grid = jet((15, 17, 13), faces)
    project(grid, GaussSeidel(0))
    compute_divergence(grid)
    multigrid = Multigrid(grid, 1, 2)
    residuals = []
    for _ in range(4):
        multigrid(grid)
        residual = host(multigrid.residual())
        residuals.append(float(np.linalg.norm(residual) / np.linalg.norm(host(grid.divergence))))
    assert residuals[-1] < 0.01
    assert all(later < 0.5 * earlier for earlier, later in zip(residuals, residuals[1:]))


def test_levels_halve_down_to_a_few_cells(cuda_device):
    from plume_b200.sim.multigrid import Multigrid, coarse_cells

    grid = cuda_grid(cells=(38, 48, 38))
    assert [level.cells for level in Multigrid(grid, 1, 2).levels] == [
        (38, 48, 38), (19, 24, 19), (10, 12, 10), (5, 6, 5), (3, 3, 3), (2, 2, 2)]
    assert coarse_cells((5, 6, 5)) == (3, 3, 3)


def test_multigrid_keeps_closed_walls_exactly_zero_and_repeats_bit_for_bit(cuda_device):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import project

    grid = jet((16, 16, 16), OPEN)
    random_velocity(grid, 3)
    project(grid, Multigrid(grid, 2, 2))
    assert np.all(host(grid.v.data)[:, 0, :] == 0.0)
    pressures = []
    for _ in range(2):
        grid = jet((15, 17, 13), OPEN)
        project(grid, Multigrid(grid, 2, 2))
        pressures.append(host(grid.pressure).tobytes())
    assert pressures[0] == pressures[1]


def test_a_tall_thin_domain_converges(cuda_device):
    from plume_b200.sim.multigrid import Multigrid

    grid = jet((6, 96, 6), ALL_CLOSED)
    assert divergence_left(grid, lambda g: Multigrid(g, 2, 2)(g)) < 0.1


# ---- forces (sim/test_forces.py) ---------------------------------------------------------------------------

def test_drag_without_wind_decays_exponentially(cuda_device):
    from plume_b200.sim.forces import apply_drag

    grid = cuda_grid()
    for value, field in zip((1.0, -2.0, 0.5), grid.velocity_fields()):
        field.data.fill_(value)
    for _ in range(10):
        apply_drag(grid, (0.0, 0.0, 0.0), 2.0, 0.05)
    decay = math.exp(-2.0 * 0.5)
    assert np.allclose(host(grid.u.data), 1.0 * decay, rtol=1e-5, atol=0.0)
    assert np.allclose(host(grid.v.data), -2.0 * decay, rtol=1e-5, atol=0.0)


def test_drag_pulls_the_gas_to_the_wind(cuda_device):
    from plume_b200.sim.forces import apply_drag

    grid = cuda_grid()
    for _ in range(100):
        apply_drag(grid, (1.5, 0.0, -0.5), 4.0, 0.05)
    assert np.abs(host(grid.u.data) - 1.5).max() <= 1e-4
    assert np.abs(host(grid.w.data) + 0.5).max() <= 1e-4


def vortex_tube(grid, core_m=0.25):
    """A counterclockwise swirl (seen from +z) around the z line through the grid's centre."""
    nx, ny, _ = grid.cells
    cell = grid.info.cell_m

    def component(shape, offset, which):
        idx = np.indices(shape).astype(np.float64)
        x = (idx[0] + offset[0]) * cell - nx * cell / 2
        y = (idx[1] + offset[1]) * cell - ny * cell / 2
        falloff = np.exp(-(x * x + y * y) / (2 * core_m * core_m))
        return (-y if which == 0 else x) * falloff / core_m

    put(grid.u.data, component(tuple(grid.u.data.shape), (0.0, 0.5), 0))
    put(grid.v.data, component(tuple(grid.v.data.shape), (0.5, 0.0), 1))


def peak_spin(grid):
    from plume_b200.sim.vorticity import VorticityConfinement

    return float(np.linalg.norm(host(VorticityConfinement(grid).measure_curl(grid)), axis=-1).max())


def test_confinement_at_zero_changes_no_bit(cuda_device):
    from plume_b200.sim.vorticity import VorticityConfinement

    grid = cuda_grid()
    vortex_tube(grid)
    before = [host(f.data).copy() for f in grid.velocity_fields()]
    VorticityConfinement(grid).apply(grid, 0.0, 0.05)
    assert all(np.array_equal(a, host(f.data)) for a, f in zip(before, grid.velocity_fields()))


def test_confinement_spins_a_vortex_up(cuda_device):
    from plume_b200.sim.vorticity import VorticityConfinement

    grid = cuda_grid()
    vortex_tube(grid)
    before = peak_spin(grid)
    confinement = VorticityConfinement(grid)
    for _ in range(10):
        confinement.apply(grid, 5.0, 0.02)
    assert peak_spin(grid) > 1.5 * before


def test_the_push_grows_with_the_cell_size(cuda_device):
    from plume_b200.sim.vorticity import VorticityConfinement

    pushes = []
    for cells, cell_m in (((32, 32, 4), 0.05), ((16, 16, 2), 0.1)):
        grid = cuda_grid(cells=cells, cell_m=cell_m)
        vortex_tube(grid)
        confinement = VorticityConfinement(grid)
        confinement.measure_curl(grid)
        confinement.apply(grid, 1.0, 0.0)
        pushes.append(float(np.linalg.norm(host(confinement.push), axis=-1).max()))
    assert 1.5 < pushes[1] / pushes[0] < 2.2


# ---- turbulence (sim/test_turbulence.py) -------------------------------------------------------------------

def turbulence_push(seed=1, time_s=0.0, cells=(16, 16, 16), cell_m=0.1, scale_m=0.4, speed_mps=0.2):
    """The face velocities one unit step of turbulence gives a grid at rest."""
    from plume_b200.sim.turbulence import apply_turbulence

    grid = cuda_grid(cells=cells, cell_m=cell_m)
    apply_turbulence(grid, seed, scale_m, 1.0, speed_mps, time_s, 1.0)
    return grid


def faces(grid):
    return [host(f.data).copy() for f in grid.velocity_fields()]


def test_zero_turbulence_changes_nothing(cuda_device):
    from plume_b200.sim.turbulence import apply_turbulence

    grid = cuda_grid()
    apply_turbulence(grid, 1, 0.4, 0.0, 0.2, 0.0, 1.0)
    assert not any(f.any() for f in faces(grid))


def test_the_turbulence_push_is_divergence_free(cuda_device):
    from plume_b200.sim.pressure import compute_divergence

    grid = turbulence_push()
    magnitude = max(np.abs(f).max() for f in faces(grid))
    divergence = np.abs(host(compute_divergence(grid))).max() * grid.info.cell_m
    assert magnitude > 0.3 and divergence < 1e-5 * magnitude


def test_the_same_seed_repeats_and_another_differs(cuda_device):
    first, again, other = (faces(turbulence_push(seed)) for seed in (1, 1, 2))
    assert all(np.array_equal(a, b) for a, b in zip(first, again))
    assert not all(np.array_equal(a, b) for a, b in zip(first, other))


def correlation(a, b):
    a = np.concatenate([f.ravel() for f in a]).astype(np.float64)
    b = np.concatenate([f.ravel() for f in b]).astype(np.float64)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))


def test_the_pattern_renews_over_scale_over_speed(cuda_device):
    start = faces(turbulence_push(time_s=0.0))  # renewal time 0.4 m / 0.2 m/s = 2 s
    assert correlation(start, faces(turbulence_push(time_s=0.05))) > 0.99
    assert correlation(start, faces(turbulence_push(time_s=2.0))) < 0.5


def test_two_cell_sizes_give_the_same_push(cuda_device):
    fine = host(turbulence_push(cells=(32, 32, 32), cell_m=0.05, scale_m=0.5).v.data)
    coarse = host(turbulence_push(cells=(16, 16, 16), cell_m=0.1, scale_m=0.5).v.data)
    # a coarse v face (i, j, k) sits at fine (2i + 0.5, 2j, 2k + 0.5): the mean of four fine faces
    matched = 0.25 * (fine[0::2, 0::2, 0::2] + fine[1::2, 0::2, 0::2] + fine[0::2, 0::2, 1::2] + fine[1::2, 0::2, 1::2])
    assert np.abs(matched - coarse).max() / np.abs(coarse).max() < 0.05


# ---- emitters (sim/test_emitters.py) -----------------------------------------------------------------------

CELL_M = 0.05


def emitted(seed=1, time_s=0.0, steps=1, dt=0.05, **emitter):
    from plume_b200.sim.emitters import emit, emitter_params

    settings = {"name": "e", "center_m": [0.0, 0.6, 0.0], "radius_m": 0.3, "end_s": 1.0, "smoke_per_s": 2.0}
    settings.update(emitter)
    recipe = tiny_recipe(seed=seed, emitter=[settings])
    grid = cuda_grid(cells=(24, 24, 24), cell_m=CELL_M)
    params = emitter_params(recipe.emitter, "cuda:0")
    for step in range(steps):
        emit(grid, params, recipe.seed, time_s + step * dt, dt)
    return grid


def test_a_sphere_emits_rate_times_volume(cuda_device):
    total = float(host(emitted(steps=20, edge_softness=0.0).smoke.data).astype(np.float64).sum()) * CELL_M**3
    assert total == pytest.approx(2.0 * 4.0 / 3.0 * math.pi * 0.3**3, rel=0.05)


def test_nothing_is_emitted_outside_the_window(cuda_device):
    assert float(emitted(time_s=1.0).smoke.data.sum()) == 0.0


def test_the_emitter_holds_its_temperature(cuda_device):
    temperature = host(emitted(temperature_k=900.0, edge_softness=0.0).temperature.data)
    assert temperature[12, 12, 12] == pytest.approx(900.0) and temperature[0, 0, 0] == pytest.approx(293.0)


def test_the_noise_repeats_with_its_seed(cuda_device):
    noisy = {"noise": {"scale_m": 0.1, "strength": 0.8}}
    first, again, other = (host(emitted(seed=seed, **noisy).smoke.data) for seed in (7, 7, 8))
    assert np.array_equal(first, again) and not np.array_equal(first, other)


def test_outward_velocity_points_away_from_the_centre(cuda_device):
    u = host(emitted(velocity_mps=[0.0, 2.0, 0.0], velocity_mode="outward", edge_softness=0.0).u.data)
    assert u[16, 12, 12] > 1.9 and u[8, 12, 12] < -1.9


def test_a_soft_edge_blends_the_same_over_one_step_or_two_halves(cuda_device):
    settings = {"temperature_k": 900.0, "velocity_mps": [0.0, 2.0, 0.0], "edge_softness": 0.8}
    one = emitted(steps=1, dt=0.05, **settings)
    two = emitted(steps=2, dt=0.025, **settings)
    edge = (12, 17, 12)  # 0.25 m above the centre: inside the 0.3 m sphere's soft edge
    assert 293.0 < host(one.temperature.data)[edge] < 900.0
    np.testing.assert_allclose(host(two.temperature.data), host(one.temperature.data), rtol=1e-5)
    np.testing.assert_allclose(host(two.v.data), host(one.v.data), rtol=1e-5, atol=1e-6)


# ---- the smoke budget and sums (sim/test_conserve.py) -----------------------------------------------------

def test_triple_sum_is_numpys_sum(cuda_device):
    import torch

    from plume_b200.sim.reduce import TripleSum

    rng = np.random.default_rng(2)
    arrays = [rng.random((5, 7, 9)).astype(np.float32) for _ in range(3)]
    sums = TripleSum((5, 7, 9), "cuda:0")(*(torch.from_numpy(a).cuda() for a in arrays))
    assert sums == pytest.approx([a.astype(np.float64).sum() for a in arrays], rel=1e-6)


def smoke_below(height_m, recipe):
    from plume_b200.recipe.derived import derive
    from plume_b200.sim.run import simulate

    rows = int(round(height_m / recipe.domain.cell_m))
    totals = []
    simulate(recipe, derive(recipe), "cuda:0",
             lambda frame, grid: totals.append(float(host(grid.smoke.data)[:, :rows, :].astype(np.float64).sum())))
    return totals


def test_an_open_top_does_not_drain_the_smoke_still_inside(cuda_device):
    puff = [{"name": "puff", "center_m": [0.0, 0.3, 0.0], "radius_m": 0.2, "end_s": 0.1, "smoke_per_s": 20.0,
             "temperature_k": 900.0}]
    short = smoke_below(0.8, tiny_recipe(domain={"size_m": [1.2, 0.8, 1.2], "cell_m": 0.05}, emitter=puff))
    tall = smoke_below(0.8, tiny_recipe(domain={"size_m": [1.2, 2.4, 1.2], "cell_m": 0.05}, emitter=puff))
    for frame, (s, t) in enumerate(zip(short, tall)):
        assert s > 0.8 * t, frame


# ---- the CFL cap and the frame loop (sim/test_step_cap.py, sim/test_frame_loop.py) -------------------------

def run(recipe, collect=lambda grid: host(grid.smoke.data).copy()):
    from plume_b200.recipe.derived import derive
    from plume_b200.sim.run import simulate

    results = []
    log = simulate(recipe, derive(recipe), "cuda:0", lambda frame, grid: results.append(collect(grid)))
    return log, results


JET = {"name": "jet", "center_m": [0.0, 0.3, 0.0], "radius_m": 0.15, "end_s": 0.5, "smoke_per_s": 5.0}


def test_a_slow_puff_keeps_its_substeps(cuda_device):
    log, _ = run(tiny_recipe())
    assert log.steps_per_frame == (3, 3, 3, 3) and log.added_steps == 0


def test_a_cap_that_never_binds_changes_no_bit(cuda_device):
    from plume_b200.recipe.derived import derive
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper

    recipe = tiny_recipe()
    derived = derive(recipe)
    _, capped = run(recipe)
    d = recipe.domain
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0")
    stepper = Stepper(grid, recipe)
    for frame in range(recipe.time.frames):
        for n in range(derived.steps_per_frame):
            stepper.step((frame * derived.steps_per_frame + n) * derived.dt_s, derived.dt_s)
        assert np.array_equal(capped[frame], host(grid.smoke.data)), frame


def test_a_fast_emitter_gets_more_steps(cuda_device):
    log, _ = run(tiny_recipe(emitter=[dict(JET, velocity_mps=[0.0, 4.0, 0.0])]))
    assert log.steps_per_frame[0] == 20  # ceil(4 m/s * 0.25 s / 0.05 m)
    assert log.steps_per_frame[1] >= 20 and all(n >= 3 for n in log.steps_per_frame) and log.added_steps > 0


def test_more_than_max_substeps_is_a_recipe_error(cuda_device):
    from plume_b200.recipe.errors import RecipeError

    jet = {k: v for k, v in JET.items() if k != "smoke_per_s"}
    with pytest.raises(RecipeError, match="max_substeps"):
        run(tiny_recipe(emitter=[dict(jet, velocity_mps=[0.0, 4.0, 0.0])], solver={"max_substeps": 10}))


def test_two_runs_choose_the_same_steps(cuda_device):
    recipe = tiny_recipe(emitter=[dict(JET, velocity_mps=[0.0, 2.0, 0.0])])
    assert run(recipe)[0] == run(recipe)[0]


def test_warmup_runs_in_blocks_of_a_frame(cuda_device, monkeypatch):
    from plume_b200.sim import step_cap

    blocks = []
    plan = step_cap.StepCap.plan

    def recording(self, grid, start_s, length_s, base_steps, label):
        blocks.append((label, base_steps))
        return plan(self, grid, start_s, length_s, base_steps, label)

    monkeypatch.setattr(step_cap.StepCap, "plan", recording)
    log, _ = run(tiny_recipe(time={"duration_s": 1.0, "frames": 4, "warmup_s": 0.6}))
    assert [base for label, base in blocks if label == "warmup"] == [3, 3, 1]  # 0.6 s at 1/12 s is 7 steps
    assert log.warmup_steps == 7 and log.total_steps == 7 + 12


CLOSED_FACES = {"faces": {"bottom": "closed", "top": "closed", "left": "closed", "right": "closed",
                          "back": "closed", "front": "closed"}}


def smoke_height(grid):
    smoke = host(grid.smoke.data).astype(np.float64)
    return float((smoke.sum(axis=(0, 2)) * (np.arange(smoke.shape[1]) + 0.5)).sum() / smoke.sum())


def test_a_hot_puff_rises(cuda_device):
    recipe = tiny_recipe(emitter=[{"name": "puff", "center_m": [0.0, 0.25, 0.0], "radius_m": 0.15, "end_s": 0.2,
                                   "smoke_per_s": 5.0, "temperature_k": 600.0}])
    _, heights = run(recipe, smoke_height)
    assert heights == sorted(heights) and heights[-1] - heights[0] > 2.0


def test_a_closed_box_nearly_conserves_smoke_and_never_gains(cuda_device):
    recipe = tiny_recipe(domain={"size_m": [1.2, 1.2, 1.2], "cell_m": 0.05, **CLOSED_FACES},
                         emitter=[{"name": "puff", "center_m": [0.0, 0.4, 0.0], "radius_m": 0.2, "end_s": 0.05,
                                   "smoke_per_s": 5.0, "temperature_k": 320.0}],
                         time={"duration_s": 2.0, "frames": 8, "substeps": 5})
    _, totals = run(recipe, lambda grid: float(host(grid.smoke.data).astype(np.float64).sum()))
    assert totals[-1] == pytest.approx(totals[0], rel=0.15) and totals[-1] <= totals[0] * (1 + 1e-5)


def test_cooling_relaxes_the_temperature_to_ambient(cuda_device):
    recipe = tiny_recipe(emitter=[{"name": "puff", "center_m": [0.0, 0.4, 0.0], "radius_m": 0.2, "end_s": 0.05,
                                   "temperature_k": 900.0}],
                         dissipation={"cooling_per_s": 3.0}, forces={"heat_buoyancy": 0.0})
    _, peaks = run(recipe, lambda grid: float(grid.temperature.data.max()))
    assert peaks == sorted(peaks, reverse=True) and peaks[-1] - 293.0 < 0.1 * (900.0 - 293.0)


def test_the_frame_generator_is_simulate(cuda_device):
    from plume_b200.recipe.derived import derive
    from plume_b200.sim.run import simulate, simulate_frames

    recipe = tiny_recipe()
    derived = derive(recipe)
    frames = simulate_frames(recipe, derived, "cuda:0")
    seen = []
    while True:
        try:
            frame, grid = next(frames)
        except StopIteration as finished:
            log = finished.value
            break
        seen.append((frame, float(host(grid.smoke.data).astype(np.float64).sum())))
    expected = []
    expected_log = simulate(recipe, derived, "cuda:0",
                            lambda frame, grid: expected.append((frame, float(host(grid.smoke.data).astype(np.float64).sum()))))
    assert [f for f, _ in seen] == [0, 1, 2, 3] and seen == expected and log == expected_log
    assert log.steps_per_frame == (derived.steps_per_frame,) * 4 and log.warmup_steps == 0
