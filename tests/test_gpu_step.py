"""Whole-substep and whole-run parity of the CUDA path (plume_step through Stepper, and the frame loop)
against the FP32 oracle. Tolerance for one substep: 1e-4 relative. With the two-pass advection kernels every
field matches to the last bit except where the emitter's pow differs by an ulp; the fused advection (the
default) blends with fused multiply-adds and agrees to about an ulp per operator."""

import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.derived import derive
from plume_b200.workloads import operator_fields, plain_step_recipe
from support import FIELDS, assert_same, host, load_state, max_rel

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
SUBSTEP_RTOL = 1e-4


def stepper_pair(recipe, seed=3):
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper

    derived = derive(recipe)
    d = recipe.domain
    o = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k)
    c = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0")
    load_state(o, c, operator_fields(derived.cells, seed, d.ambient_k))
    return o, c, O.Stepper(o, recipe), Stepper(c, recipe), derived


def compare_fields(o, c, rtol, what):
    worst = {}
    for name in FIELDS:
        worst[name] = max_rel(host(getattr(c, name).data), getattr(o, name).data, floor=1e-2)
        assert worst[name] < rtol, f"{what}: {name} differs by {worst[name]:.3g}"
    worst["pressure"] = max_rel(host(c.pressure), o.pressure, floor=1e-6)
    return worst


@pytest.mark.parametrize("cells", [(32, 48, 32), (19, 24, 17)])
def test_one_substep_matches_the_oracle(cuda_device, cells):
    recipe = plain_step_recipe(cells, cycles=4)
    o, c, os_, cs, derived = stepper_pair(recipe)
    os_.step(0.0, derived.dt_s)
    cs.step(0.0, derived.dt_s)
    compare_fields(o, c, SUBSTEP_RTOL, "one substep")


@pytest.mark.parametrize("cells,faces", [((19, 24, 17), None), ((16, 12, 20), "closed"), ((2, 3, 1), None)],
                         ids=["19x24x17-open", "16x12x20-closed", "2x3x1-open"])
@pytest.mark.parametrize("fused", [False, True], ids=["two-pass", "fused"])
def test_a_substep_without_exp_or_pow_gives_the_oracles_floats(cuda_device, cells, faces, fused):
    """With the emitter finished and no drag or dissipation, no operator of the substep calls exp or pow, so
    with the two-pass advection every field, the pressure included, is the oracle's to the last bit: the
    step's velocity advection (the three face arrays in one launch) and its smoke and temperature advection,
    walls included. The fused advection gives the same substep within the substep tolerance."""
    import dataclasses

    from plume_b200 import _native as N

    recipe = plain_step_recipe(cells, cycles=2)
    recipe = dataclasses.replace(
        recipe, emitter=[dataclasses.replace(recipe.emitter[0], end_s=0.01)],
        forces=dataclasses.replace(recipe.forces, drag_per_s=0.0),
        dissipation=dataclasses.replace(recipe.dissipation, smoke_per_s=0.0, cooling_per_s=0.0))
    if faces == "closed":
        recipe = dataclasses.replace(recipe, domain=dataclasses.replace(
            recipe.domain, faces=dataclasses.replace(recipe.domain.faces, **{
                f.name: "closed" for f in dataclasses.fields(recipe.domain.faces)})))
    o, c, os_, cs, derived = stepper_pair(recipe)
    os_.step(1.0, derived.dt_s)
    N.call("plume_use_fused_advection", 3 if fused else 0)  # both fused passes, or neither
    try:
        cs.step(1.0, derived.dt_s)
    finally:
        N.call("plume_use_fused_advection", 1)
    if fused:
        compare_fields(o, c, SUBSTEP_RTOL, "fused substep")
        return
    for name in FIELDS:
        assert_same(host(getattr(c, name).data), getattr(o, name).data, name)
    assert_same(host(c.pressure), o.pressure, "pressure")


def test_eight_substeps_with_turbulence_and_dissipation_match_the_oracle(cuda_device):
    import dataclasses

    recipe = plain_step_recipe((24, 32, 24), cycles=2)
    recipe = dataclasses.replace(
        recipe, forces=dataclasses.replace(recipe.forces, turbulence=dataclasses.replace(
            recipe.forces.turbulence, strength_mps2=0.3, scale_m=0.1)),
        dissipation=dataclasses.replace(recipe.dissipation, smoke_per_s=1.6, cooling_per_s=1.0))
    o, c, os_, cs, derived = stepper_pair(recipe)
    for n in range(8):
        os_.step(n * derived.dt_s, derived.dt_s)
        cs.step(n * derived.dt_s, derived.dt_s)
    compare_fields(o, c, SUBSTEP_RTOL, "eight substeps")


def test_gauss_seidel_substep_matches_the_oracle(cuda_device):
    import dataclasses

    recipe = plain_step_recipe((16, 24, 16))
    recipe = dataclasses.replace(recipe, solver=dataclasses.replace(recipe.solver, pressure_solver="gauss_seidel",
                                                                    pressure_iterations=30))
    o, c, os_, cs, derived = stepper_pair(recipe)
    os_.step(0.0, derived.dt_s)
    cs.step(0.0, derived.dt_s)
    compare_fields(o, c, SUBSTEP_RTOL, "Gauss-Seidel substep")


def test_smoke_puff_preview_run_matches_the_oracle(cuda_device):
    """The reference's smoke puff preview (38 x 48 x 38, 16 frames, 192 substeps) through the CUDA frame loop
    and renderer: raw frames within 1e-3 of the oracle's (chaotic flow; the emitter's pow differs by an ulp),
    per-frame channel sums within 0.5% of the golden statistics, and identical step counts."""
    from plume_b200.recipe.load import load_recipe
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.run import simulate

    recipe = load_recipe(GOLDEN / "smoke_puff.toml", preview=True)
    derived = derive(recipe)
    view = sheet_domain_view(recipe, derived)
    renderer = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "cuda:0")
    frames = []
    log = simulate(recipe, derived, "cuda:0", lambda frame, grid: frames.append(renderer.render(grid)))
    stats = json.loads((GOLDEN / "preview_raw_stats.json").read_text())
    assert list(log.steps_per_frame) == stats["steps_per_frame"]
    oracle_renderer = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels)
    expected = []
    O.simulate(recipe, derived, lambda frame, grid: expected.append(oracle_renderer.render(grid)))
    for index, (frame, reference) in enumerate(zip(frames, expected)):
        assert np.abs(frame - reference).max() < 1e-3, f"frame {index}"
        sums = frame.astype(np.float64).sum(axis=(0, 1))
        for channel in (1, 2):  # thickness and shade * thickness
            golden = stats["sum"][index][channel]
            assert abs(sums[channel] - golden) <= 5e-3 * abs(golden), f"frame {index} channel {channel}"


def test_same_input_gives_identical_bytes(cuda_device):
    """Every kernel is a gather with a fixed order: two runs of the same substeps give identical bytes."""
    results = []
    for _ in range(2):
        recipe = plain_step_recipe((24, 32, 24), cycles=2)
        _, c, _, cs, derived = stepper_pair(recipe)
        for n in range(4):
            cs.step(n * derived.dt_s, derived.dt_s)
        results.append(b"".join(host(getattr(c, name).data).tobytes() for name in FIELDS))
    assert results[0] == results[1]


def test_a_substep_with_the_split_top_level_gives_the_oracles_floats(cuda_device):
    """plume_step with the pressure solve's top level in colour-split storage (forced on at this size) and the
    two-pass advection: no exp or pow in the substep, so every field and the pressure are the oracle's."""
    import dataclasses

    from plume_b200 import _native as N

    recipe = plain_step_recipe((21, 24, 19), cycles=2)
    recipe = dataclasses.replace(
        recipe, emitter=[dataclasses.replace(recipe.emitter[0], end_s=0.01)],
        forces=dataclasses.replace(recipe.forces, drag_per_s=0.0),
        dissipation=dataclasses.replace(recipe.dissipation, smoke_per_s=0.0, cooling_per_s=0.0))
    o, c, os_, cs, derived = stepper_pair(recipe)
    os_.step(1.0, derived.dt_s)
    default = N.lib().plume_split_min_cells()
    N.call("plume_use_fused_advection", 0)
    N.call("plume_tune_split", 1)
    try:
        cs.step(1.0, derived.dt_s)
    finally:
        N.call("plume_use_fused_advection", 1)
        N.call("plume_tune_split", default)
    for name in FIELDS:
        assert_same(host(getattr(c, name).data), getattr(o, name).data, name)
    assert_same(host(c.pressure), o.pressure, "pressure")
