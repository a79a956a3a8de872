"""The adjoint through the velocity path (FlowFit): the gradient of the rendered-thickness loss with respect to
heat_buoyancy and drag_per_s, whose effect reaches the smoke only through the velocity (buoyancy, drag,
self-advection, projection, scalar advection), and with respect to the source field, with a smoke weight so
that the smoke also pushes the velocity.

Checks: each scalar's gradient against central differences of the FP64 oracle's loss (h = 1e-3; measured
agreement 3e-3 and 4e-3) and, more loosely, of the float32 model's own loss (h = 1e-2, whose rounding and
curvature put it a few percent off); the source gradient against central differences on the voxels with the
largest gradient; and, without smoke weight, the source gradient equals SourceFit's (the smoke-only adjoint)
where the velocity path adds nothing. A second run adds vorticity confinement and curl-noise turbulence, and
checks the confinement strength's gradient as well."""

import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.derived import derive
from plume_b200.workloads import plain_step_recipe

pytestmark = pytest.mark.gpu

CELLS = (20, 28, 20)
SOURCE = (5, 5, 5)
CORNER = (7, 2, 7)
SUBSTEPS = 10
CYCLES = 8  # forward V-cycles: the forward projection close to exact, as the adjoint's is
SCALAR_RTOL_FP64 = 1e-2  # against FP64 central differences
SCALAR_RTOL = 6e-2       # against float32 central differences
SOURCE_RTOL = 2e-2


def flow_recipe(smoke_weight=0.05, **forces):
    recipe = plain_step_recipe(CELLS, cycles=CYCLES, frames=4, substeps=3)
    f = dataclasses.replace(recipe.forces, vorticity_confinement=0.0, smoke_weight=smoke_weight, **forces)
    return dataclasses.replace(recipe, forces=f, dissipation=dataclasses.replace(
        recipe.dissipation, smoke_per_s=0.3, cooling_per_s=0.2))


def oracle_loss(recipe, source, target, precision="f64"):
    derived = derive(recipe)
    d = recipe.domain

    def add(grid, time_s, dt):
        grid.smoke.data[CORNER[0]:CORNER[0] + SOURCE[0], CORNER[1]:CORNER[1] + SOURCE[1],
                        CORNER[2]:CORNER[2] + SOURCE[2]] += source * dt

    grid = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k, precision)
    stepper = O.Stepper(grid, recipe, before_step=add)
    for n in range(SUBSTEPS):
        stepper.step(n * derived.dt_s, derived.dt_s)
    from plume_b200.render.camera import sheet_domain_view

    view = sheet_domain_view(recipe, derived)
    thickness = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels,
                                precision).render(grid)[..., 1]
    return float(((thickness - target) ** 2).sum()), thickness


@pytest.fixture(scope="module")
def case():
    import torch

    from plume_b200.adjoint import FlowFit

    recipe = flow_recipe()
    rng = np.random.default_rng(4)
    source = rng.uniform(0.0, 1.0, SOURCE) * 20.0
    target_recipe = dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, heat_buoyancy=1.2))
    _, target = oracle_loss(target_recipe, np.clip(source + rng.normal(0.0, 4.0, SOURCE), 0.0, None), 0.0)
    fit = FlowFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4, adjoint_cycles=12)
    src = torch.from_numpy(source.astype(np.float32))
    tgt = torch.from_numpy(target.astype(np.float32))
    loss, grad, scalars, _ = fit.loss_and_grad(src, tgt)
    return recipe, source, target, fit, src, tgt, loss, grad.cpu().numpy().astype(np.float64), scalars


@pytest.mark.parametrize("name,h", [("heat_buoyancy", 1e-2), ("drag_per_s", 1e-2)])
def test_scalar_gradients_match_central_differences(cuda_device, case, name, h):
    recipe, source, target, fit, src, tgt, loss, _, scalars = case
    value = getattr(recipe.forces, name)
    up = fit.with_forces(**{name: value + h}).loss(src, tgt)
    down = fit.with_forces(**{name: value - h}).loss(src, tgt)
    fd = (up - down) / (2.0 * h)
    up64, _ = oracle_loss(dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, **{name: value + 1e-3})),
                          source, target)
    down64, _ = oracle_loss(dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, **{name: value - 1e-3})),
                            source, target)
    fd64 = (up64 - down64) / 2e-3
    print(f"{name}: adjoint {scalars[name]:.6g}  float32 FD {fd:.6g}  FP64 FD {fd64:.6g}")
    assert abs(scalars[name] - fd) <= SCALAR_RTOL * abs(fd)
    assert abs(scalars[name] - fd64) <= SCALAR_RTOL_FP64 * abs(fd64)


def test_source_gradient_matches_central_differences(cuda_device, case):
    import torch

    _, source, target, fit, src, tgt, _, grad, _ = case
    scale = float(np.abs(grad).max())
    picks = list(np.argsort(np.abs(grad).ravel())[-4:])
    h = 2e-2 * float(source.max())
    errors = []
    for flat in picks:
        index = np.unravel_index(flat, SOURCE)
        up, down = source.copy(), source.copy()
        up[index] += h
        down[index] -= h
        fd = (fit.loss(torch.from_numpy(up.astype(np.float32)), tgt) -
              fit.loss(torch.from_numpy(down.astype(np.float32)), tgt)) / (2.0 * h)
        errors.append(abs(grad[index] - fd) / scale)
    print("source gradient errors (of the gradient's scale):", [f"{e:.2e}" for e in errors])
    assert max(errors) <= SOURCE_RTOL


def test_without_smoke_weight_the_source_gradient_is_the_smoke_adjoints(cuda_device):
    import torch

    from plume_b200.adjoint import FlowFit, SourceFit

    recipe = flow_recipe(smoke_weight=0.0)
    rng = np.random.default_rng(6)
    source = torch.from_numpy((rng.uniform(0.0, 1.0, SOURCE) * 20.0).astype(np.float32))
    derived = derive(recipe)
    from plume_b200.render.camera import sheet_domain_view

    view = sheet_domain_view(recipe, derived)
    target = torch.full((view.height_px, view.width_px), 0.1, dtype=torch.float32)
    _, flow_grad, scalars, _ = FlowFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4).loss_and_grad(
        source, target)
    _, smoke_grad, _ = SourceFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4).loss_and_grad(
        source, target)
    a, b = flow_grad.cpu().numpy(), smoke_grad.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max()
    assert all(np.isfinite(v) for v in scalars.values())


WARM_RTOL = 1e-5  # the warm-started 4-cycle adjoint solve against 12 cycles, on each gradient (measured 3e-7)


def test_a_warm_started_adjoint_solve_of_four_cycles_gives_the_same_gradients(cuda_device, case):
    """The adjoint projection solved by 4 V-cycles from the adjoint pressure of the substep after (the default
    for a recipe of 4 cycles) against the case's 12 cycles: the gradients agree within WARM_RTOL, so the
    cheaper solve keeps the finite-difference agreement above."""
    from plume_b200.adjoint import FlowFit

    recipe, _, _, _, src, tgt, loss, grad, scalars = case
    fit = FlowFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4, adjoint_cycles=4)
    assert fit.warm_start
    warm_loss, warm_grad, warm_scalars, _ = fit.loss_and_grad(src, tgt)
    assert warm_loss == loss
    warm_grad = warm_grad.cpu().numpy().astype(np.float64)
    source_err = float(np.abs(warm_grad - grad).max()) / float(np.abs(grad).max())
    print("warm start: source", f"{source_err:.2e}",
          {name: f"{abs(warm_scalars[name] - scalars[name]) / abs(scalars[name]):.2e}" for name in scalars})
    assert source_err <= WARM_RTOL
    for name in scalars:
        assert abs(warm_scalars[name] - scalars[name]) <= WARM_RTOL * abs(scalars[name])


def test_the_tape_budget_changes_the_time_not_the_gradient(cuda_device, case):
    """With no tape budget every segment is recomputed from its checkpoint; the case's run (the default budget)
    kept every record from its forward pass. The gradients agree to the atomics' run-to-run rounding."""
    from plume_b200.adjoint import FlowFit

    recipe, _, _, fit, src, tgt, loss, grad, scalars = case
    assert fit._taped_from() == 0  # the default budget holds this run's whole tape
    lean = FlowFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4, adjoint_cycles=12, tape_bytes=0)
    assert lean._taped_from() == SUBSTEPS
    lean_loss, lean_grad, lean_scalars, _ = lean.loss_and_grad(src, tgt)
    assert lean_loss == loss
    lean_grad = lean_grad.cpu().numpy().astype(np.float64)
    assert float(np.abs(lean_grad - grad).max()) <= 1e-6 * float(np.abs(grad).max())
    for name in scalars:
        assert abs(lean_scalars[name] - scalars[name]) <= 1e-6 * abs(scalars[name])


@pytest.fixture(scope="module")
def confined_case():
    """The case's run with vorticity confinement (0.3) and curl-noise turbulence on."""
    import torch

    from plume_b200.adjoint import FlowFit

    base = flow_recipe()
    turbulence = dataclasses.replace(base.forces.turbulence, strength_mps2=0.4, scale_m=0.15, speed_mps=0.1)
    recipe = dataclasses.replace(base, forces=dataclasses.replace(base.forces, vorticity_confinement=0.3,
                                                                   turbulence=turbulence))
    rng = np.random.default_rng(5)
    source = rng.uniform(0.0, 1.0, SOURCE) * 20.0
    target_recipe = dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, heat_buoyancy=1.2,
                                                                           vorticity_confinement=0.4))
    _, target = oracle_loss(target_recipe, np.clip(source + rng.normal(0.0, 4.0, SOURCE), 0.0, None), 0.0)
    fit = FlowFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=4, adjoint_cycles=12)
    src = torch.from_numpy(source.astype(np.float32))
    tgt = torch.from_numpy(target.astype(np.float32))
    loss, grad, scalars, _ = fit.loss_and_grad(src, tgt)
    return recipe, source, target, fit, src, tgt, loss, grad.cpu().numpy().astype(np.float64), scalars


# The confinement strength's gradient is small in this run (the loss barely moves with it): against FP64 central
# differences it agrees to 2.7% (3.1e-7 absolute, less than the other scalars' absolute gaps, which come from the
# float32 run's trajectory departing from the FP64 one), and float32 central differences of its loss are
# dominated by the loss's rounding (a 79% gap measured), so only the FP64 comparison is made for it. The
# operator itself is checked exactly in test_gpu_confinement_adjoint.py.
CONFINED_RTOL_FP64 = {"heat_buoyancy": SCALAR_RTOL_FP64, "drag_per_s": SCALAR_RTOL_FP64,
                      "vorticity_confinement": 5e-2}


@pytest.mark.parametrize("name,h", [("heat_buoyancy", 1e-2), ("drag_per_s", 1e-2), ("vorticity_confinement", None)])
def test_with_confinement_and_turbulence_the_scalar_gradients_match_central_differences(cuda_device, confined_case,
                                                                                        name, h):
    recipe, source, target, fit, src, tgt, loss, _, scalars = confined_case
    assert set(scalars) == {"heat_buoyancy", "drag_per_s", "vorticity_confinement"}
    value = getattr(recipe.forces, name)
    fd = None
    if h is not None:
        fd = (fit.with_forces(**{name: value + h}).loss(src, tgt) -
              fit.with_forces(**{name: value - h}).loss(src, tgt)) / (2.0 * h)
    moved = [oracle_loss(dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, **{name: x})), source,
                         target)[0] for x in (value + 1e-3, value - 1e-3)]
    fd64 = (moved[0] - moved[1]) / 2e-3
    print(f"{name} (confinement + turbulence): adjoint {scalars[name]:.6g}  float32 FD {fd}  FP64 FD {fd64:.6g}")
    if fd is not None:
        assert abs(scalars[name] - fd) <= SCALAR_RTOL * abs(fd)
    assert abs(scalars[name] - fd64) <= CONFINED_RTOL_FP64[name] * abs(fd64)


def test_with_confinement_and_turbulence_the_source_gradient_matches_central_differences(cuda_device, confined_case):
    import torch

    _, source, target, fit, src, tgt, _, grad, _ = confined_case
    scale = float(np.abs(grad).max())
    h = 2e-2 * float(source.max())
    errors = []
    for flat in list(np.argsort(np.abs(grad).ravel())[-4:]):
        index = np.unravel_index(flat, SOURCE)
        up, down = source.copy(), source.copy()
        up[index] += h
        down[index] -= h
        fd = (fit.loss(torch.from_numpy(up.astype(np.float32)), tgt) -
              fit.loss(torch.from_numpy(down.astype(np.float32)), tgt)) / (2.0 * h)
        errors.append(abs(grad[index] - fd) / scale)
    print("source gradient errors with confinement (of the gradient's scale):", [f"{e:.2e}" for e in errors])
    assert max(errors) <= SOURCE_RTOL
