"""Parity at the benchmark configurations, against the FP32 oracle (the restatement of the reference's Warp CPU
path), on the same inputs.

C1, the smoke puff: 64 x 96 x 64 cells, 48 frames at 24 fps, CFL 1 with at most 4 substeps, 4 V-cycles, glow
from the ambient temperature so the heat channel is exercised. Whole runs of a chaotic flow are compared as
the reference compares its CPU and GPU runs (tests/cli/test_cpu_gpu.py:27-33 in chadmv/plume): per frame,
coverage, mean and total thickness within 2%; sheet bytes within 3 (thickness) and 6 (the other channels);
and, with the golden-numbers tolerances (tests/cli/test_golden_numbers.py:148-188), heat within 0.02 and the
covered box within 0.02 of the frame. Step counts per frame are identical.

C2, the operator case: 128 x 192 x 128 seeded fields. One call of each operator within 1e-5 relative (the
largest difference over the field's largest magnitude); the multigrid solve bit for bit (no fused operations on that path) and,
refined by defect correction, to a relative residual below 1e-6; a 256 x 256 march within 1e-4; then 96 plain
substeps, compared on the smoke and temperature totals, the kinetic energy and a rendered frame's coverage,
mean and total thickness."""

import dataclasses
import math
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import sheet as S
from plume_b200 import _native as N
from plume_b200.recipe.derived import derive
from plume_b200.render.camera import sheet_domain_view
from plume_b200.workloads import operator_fields, plain_step_recipe, smoke_puff_recipe
from support import FIELDS, assert_same, host, load_state

pytestmark = pytest.mark.gpu

AMOUNT_RTOL = 0.02   # coverage, mean and total thickness (test_cpu_gpu.py:33)
HEAT_ATOL = 0.02     # mean and peak heat, box edges (test_golden_numbers.py)
SHEET_THICKNESS_BYTES = 3
SHEET_OTHER_BYTES = 6
OP_RTOL = 1e-5


def close_amount(a, b):
    return abs(a - b) <= max(AMOUNT_RTOL * abs(b), 1e-3)


def compare_frame_numbers(got_frames, want_frames):
    problems = []
    for index, (g, w) in enumerate(zip(got_frames, want_frames)):
        gc, gbox, gheat, gmean, gtotal, gpeak = S.measure_frame(g)
        wc, wbox, wheat, wmean, wtotal, wpeak = S.measure_frame(w)
        for name, a, b in (("coverage", gc, wc), ("mean_thick", gmean, wmean), ("total_thick", gtotal, wtotal)):
            if not close_amount(a, b):
                problems.append(f"frame {index} {name}: {a:.5g} vs {b:.5g}")
        for name, a, b in (("mean_heat", gheat, wheat), ("peak_heat", gpeak, wpeak)):
            if abs(a - b) > HEAT_ATOL:
                problems.append(f"frame {index} {name}: {a:.5g} vs {b:.5g}")
        if (gbox is None) != (wbox is None) or (
                gbox is not None and max(abs(x - y) for x, y in zip(gbox, wbox)) > HEAT_ATOL):
            problems.append(f"frame {index} box: {gbox} vs {wbox}")
    return problems


def test_c1_smoke_puff_run_matches_the_oracle(cuda_device):
    from plume_b200.run import run_recipe

    O.set_threads(os.cpu_count() or 1)
    recipe = smoke_puff_recipe()
    derived = derive(recipe)
    assert derived.cells == (64, 96, 64) and recipe.time.frames == 48
    assert recipe.render.glow_start_k == recipe.domain.ambient_k  # heat on
    run = run_recipe(recipe, "smoke_puff_c1")
    view = sheet_domain_view(recipe, derived)
    renderer = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels)
    raw = []
    log = O.simulate(recipe, derived, lambda frame, grid: raw.append(renderer.render(grid)))
    assert list(run.steps.steps_per_frame) == list(log.steps_per_frame)
    assert run.steps.total_steps == log.total_steps
    want, crop, margin, heat_divisor, shade_divisor = S.assemble(raw, recipe.output.frame_px, recipe.render,
                                                                 recipe.output.channels)
    got = run.assembled.frames
    assert max(float(np.asarray(f)[..., 0].max()) for f in want) > 0  # the heat channel glows
    assert compare_frame_numbers(got, want) == []
    assert abs(run.assembled.heat_divisor - heat_divisor) <= 0.02 * heat_divisor
    got_crop = (run.assembled.crop.left, run.assembled.crop.top, run.assembled.crop.side)
    if got_crop == crop:
        sheet = host(run.sheet).astype(int)
        expected = S.pack(want, recipe.output.columns).astype(int)
        assert sheet.shape == expected.shape
        assert np.abs(sheet[..., 1] - expected[..., 1]).max() <= SHEET_THICKNESS_BYTES
        others = [c for c in range(sheet.shape[-1]) if c != 1]
        assert np.abs(sheet[..., others] - expected[..., others]).max() <= SHEET_OTHER_BYTES
    else:  # the crop follows the content box; a box a pixel apart moves every byte, so compare the crop
        assert max(abs(a - b) for a, b in zip(got_crop, crop)) <= 0.02 * crop[2]


C2_CELLS = (128, 192, 128)


def c2_pair():
    from plume_b200.sim.grid import make_grid

    recipe = plain_step_recipe(C2_CELLS, cycles=4)
    derived = derive(recipe)
    d = recipe.domain
    o = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k)
    c = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0")
    load_state(o, c, operator_fields(derived.cells, 20261203, d.ambient_k))
    return recipe, derived, o, c


def check(actual, expected, what):
    """The relative error of an operator's output field: largest difference over the field's largest magnitude."""
    scale = float(np.abs(expected).max()) or 1.0
    err = float(np.abs(np.asarray(actual, np.float64) - expected).max()) / scale
    assert err < OP_RTOL, f"{what}: {err:.3g}"


def test_c2_operators_match_the_oracle(cuda_device):
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.forces import apply_buoyancy
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence
    from plume_b200.sim.vorticity import VorticityConfinement

    O.set_threads(os.cpu_count() or 1)
    recipe, derived, o, c = c2_pair()
    dt = 1.0 / 96.0
    # MacCormack of the five fields (the fused passes)
    velocity = tuple(f.data for f in o.velocity_fields())
    for name in FIELDS:
        O.advect_maccormack(getattr(o, name), velocity, o, dt)
    out = {name: torch.empty_like(getattr(c, name).data) for name in FIELDS}
    N.call("plume_maccormack_velocity", c.info, *(N.ptr(getattr(c, n).data) for n in ("u", "v", "w")),
           *(N.ptr(out[n]) for n in ("u", "v", "w")), dt / c.info.cell_m, N.stream())
    scratch = torch.empty(N.lib().plume_maccormack_scratch_floats(c.info), dtype=torch.float32, device="cuda:0")
    sums = torch.empty(N.lib().plume_smoke_scratch_doubles(c.info), dtype=torch.float64, device="cuda:0")
    N.call("plume_maccormack_scalars", c.info, *(N.ptr(f.data) for f in c.velocity_fields()), N.ptr(c.smoke.data),
           N.ptr(c.temperature.data), N.ptr(out["smoke"]), N.ptr(out["temperature"]), dt / c.info.cell_m, 0.0,
           recipe.domain.ambient_k, 1, N.ptr(scratch), N.ptr(sums, torch.float64), None, N.stream())
    for name in FIELDS:
        check(host(out[name]), getattr(o, name).next, f"MacCormack {name}")
    # buoyancy + vorticity confinement: no exp or pow, the oracle's floats
    f, d = recipe.forces, recipe.domain
    O.apply_buoyancy(o, f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, d.ambient_k, dt)
    apply_buoyancy(c, f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, d.ambient_k, dt)
    O.VorticityConfinement(o).apply(o, f.vorticity_confinement, dt)
    VorticityConfinement(c).apply(c, f.vorticity_confinement, dt)
    for name in ("u", "v", "w"):
        assert_same(host(getattr(c, name).data), getattr(o, name).data, f"forces {name}")
    # the projection's solve: 4 V-cycles bit for bit, then refined to a relative residual of 1e-6
    O.compute_divergence(o)
    compute_divergence(c)
    o.pressure[...] = 0.0
    c.pressure.zero_()
    O.Multigrid(o, 4, 2)(o)
    multigrid = Multigrid(c, 4, 2)
    multigrid(c)
    assert_same(host(c.pressure), o.pressure, "4-cycle pressure")
    c.pressure.zero_()
    refinement = multigrid.refine(c, rel_tol=1e-6)
    assert refinement.ratio <= 1e-6
    # a 256 x 256 orthographic march
    view = sheet_domain_view(recipe, derived)
    extent = max(view.width_px, view.height_px) * view.pixel_m
    view = dataclasses.replace(view, pixel_m=extent / 256, width_px=256, height_px=256)
    frame = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "cuda:0").render(c)
    expected = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels).render(o)
    assert frame.shape == (256, 256, 5)
    assert np.abs(frame[..., 1:] - expected[..., 1:]).max() < 1e-4
    heat_scale = max(float(np.abs(expected[..., 0]).max()), 1e-30)
    assert np.abs(frame[..., 0] - expected[..., 0]).max() / heat_scale < 1e-4


def test_c2_96_plain_substeps_match_the_oracle(cuda_device):
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.stepper import Stepper

    O.set_threads(os.cpu_count() or 1)
    recipe, derived, o, c = c2_pair()
    dt = derived.dt_s
    assert math.isclose(dt, 1.0 / 96.0)
    ostep, cstep = O.Stepper(o, recipe), Stepper(c, recipe)
    for n in range(96):
        ostep.step(n * dt, dt)
        cstep.step(n * dt, dt)
    for name in ("smoke", "temperature"):
        a = float(host(getattr(c, name).data).astype(np.float64).sum())
        b = float(getattr(o, name).data.astype(np.float64).sum())
        assert abs(a - b) <= 1e-3 * abs(b), f"{name} total {a} vs {b}"
    energy = [sum(float((np.asarray(x, dtype=np.float64) ** 2).sum()) for x in grid)
              for grid in ([host(f.data) for f in c.velocity_fields()], [f.data for f in o.velocity_fields()])]
    assert abs(energy[0] - energy[1]) <= AMOUNT_RTOL * energy[1]
    view = sheet_domain_view(recipe, derived)
    frame = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "cuda:0").render(c)
    expected = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels).render(o)
    thickness, want = frame[..., 1].astype(np.float64), expected[..., 1].astype(np.float64)
    assert close_amount(thickness.sum(), want.sum())
    assert close_amount(float((thickness >= 8 / 255).mean()), float((want >= 8 / 255).mean()))
    covered = want >= 8 / 255
    assert close_amount(float(thickness[covered].mean()), float(want[covered].mean()))
