"""The source-field adjoint (float32) against the FP64 oracle of the same model: its final thickness within
2e-3 and its loss within 5e-3 relative (the float32 run's own drift from FP64 over 12 substeps; the loss is a
sum of squared differences), its thickness exactly the renderer's, and its gradient against central finite
differences of the FP64 oracle's loss (h = 1e-3) within GRAD_RTOL of the gradient's scale, on the voxels with
the largest gradient and random others."""

import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.derived import derive
from plume_b200.workloads import plain_step_recipe

pytestmark = pytest.mark.gpu

CELLS = (24, 32, 24)
SOURCE = (6, 6, 6)
CORNER = (9, 3, 9)
SUBSTEPS = 12
FD_H = 1e-3
FD_H_F32 = 2e-2  # large enough that the float32 loss difference stands well above its rounding
GRAD_RTOL = 1e-3
GRAD_RTOL_FP64 = 1e-2


def adjoint_recipe():
    recipe = plain_step_recipe(CELLS, cycles=4, frames=4, substeps=3)
    forces = dataclasses.replace(recipe.forces, smoke_weight=0.0)
    return dataclasses.replace(recipe, forces=forces,
                               dissipation=dataclasses.replace(recipe.dissipation, smoke_per_s=0.4, cooling_per_s=0.2))


def oracle_loss(recipe, source, target) -> float:
    derived = derive(recipe)
    d = recipe.domain

    def add(grid, time_s, dt):
        box = grid.smoke.data[CORNER[0]:CORNER[0] + SOURCE[0], CORNER[1]:CORNER[1] + SOURCE[1],
                              CORNER[2]:CORNER[2] + SOURCE[2]]
        box += source * dt

    grid = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k, "f64")
    stepper = O.Stepper(grid, recipe, before_step=add)
    for n in range(SUBSTEPS):
        stepper.step(n * derived.dt_s, derived.dt_s)
    from plume_b200.render.camera import sheet_domain_view

    view = sheet_domain_view(recipe, derived)
    thickness = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "f64").render(grid)[..., 1]
    return float(((thickness - target) ** 2).sum()), thickness


@pytest.fixture(scope="module")
def case():
    import torch

    from plume_b200.adjoint import SourceFit

    recipe = adjoint_recipe()
    rng = np.random.default_rng(8)
    source = rng.uniform(0.0, 1.0, SOURCE) * 20.0
    target_source = np.clip(source + rng.normal(0.0, 4.0, SOURCE), 0.0, None)
    _, target = oracle_loss(recipe, target_source, 0.0)
    fit = SourceFit(recipe, SOURCE, CORNER, SUBSTEPS, "cuda:0", checkpoint_every=5)
    loss, grad, thickness = fit.loss_and_grad(torch.from_numpy(source.astype(np.float32)),
                                              torch.from_numpy(target.astype(np.float32)))
    return recipe, source, target, fit, loss, grad.cpu().numpy().astype(np.float64), thickness.cpu().numpy()


def test_loss_and_thickness_match_the_oracle(cuda_device, case):
    import torch

    from plume_b200.render.frame_renderer import FrameRenderer

    recipe, source, target, fit, loss, _, thickness = case
    want, want_thickness = oracle_loss(recipe, source, target)
    print(f"loss {loss:.6g} oracle {want:.6g}; thickness error {np.abs(thickness - want_thickness).max():.2e}")
    assert abs(loss - want) <= 5e-3 * want
    assert np.abs(thickness - want_thickness).max() < 2e-3
    grid, _ = fit.forward(torch.from_numpy(source.astype(np.float32)).cuda())
    frame = FrameRenderer(fit.view, recipe.render, grid.cells, recipe.output.channels, "cuda:0").render(grid)
    assert np.array_equal(frame[..., 1], thickness)  # the adjoint's march is the renderer's


def fd_picks(grad):
    rng = np.random.default_rng(2)
    flat = np.argsort(-np.abs(grad).ravel())
    return [np.unravel_index(i, SOURCE) for i in list(flat[:6]) + list(rng.choice(flat[6:], 6, replace=False))]


def test_gradient_matches_central_differences_of_the_same_model(cuda_device, case):
    """Central differences of the float32 model's own loss (the GPU forward): the adjoint's consistency."""
    import torch

    _, source, target, fit, _, grad, _ = case
    scale = np.abs(grad).max()
    target_t = torch.from_numpy(target.astype(np.float32))
    errors = []
    for voxel in fd_picks(grad):
        up, down = source.copy(), source.copy()
        up[voxel] += FD_H_F32
        down[voxel] -= FD_H_F32
        fd = (fit.loss(torch.from_numpy(up.astype(np.float32)), target_t)
              - fit.loss(torch.from_numpy(down.astype(np.float32)), target_t)) / (2 * FD_H_F32)
        errors.append(abs(grad[voxel] - fd) / scale)
        print(voxel, f"adjoint {grad[voxel]:.6e} float32 fd {fd:.6e} diff/scale {errors[-1]:.2e}")
    assert max(errors) <= GRAD_RTOL, max(errors)


def test_gradient_matches_central_differences_of_the_fp64_oracle(cuda_device, case):
    """Central differences of the FP64 oracle's loss: the float32 model against the plain method in double."""
    recipe, source, target, _, _, grad, _ = case
    scale = np.abs(grad).max()
    errors = []
    for voxel in fd_picks(grad):
        up, down = source.copy(), source.copy()
        up[voxel] += FD_H
        down[voxel] -= FD_H
        fd = (oracle_loss(recipe, up, target)[0] - oracle_loss(recipe, down, target)[0]) / (2 * FD_H)
        errors.append(abs(grad[voxel] - fd) / scale)
        print(voxel, f"adjoint {grad[voxel]:.6e} fp64 fd {fd:.6e} diff/scale {errors[-1]:.2e}")
    assert max(errors) <= GRAD_RTOL_FP64, max(errors)


def test_autograd_function_gives_the_same_gradient(cuda_device, case):
    import torch

    from plume_b200.adjoint import ThicknessLoss

    _, source, target, fit, loss, grad, _ = case
    s = torch.from_numpy(source.astype(np.float32)).cuda().requires_grad_(True)
    value = ThicknessLoss.apply(s, fit, torch.from_numpy(target.astype(np.float32)))
    value.backward()
    assert abs(value.item() - loss) <= 1e-6 * loss
    assert np.allclose(s.grad.cpu().numpy(), grad, rtol=1e-4, atol=1e-6 * np.abs(grad).max())


def test_force_scalar_gradients_match_central_differences_of_the_fp64_oracle(cuda_device, case):
    """d loss / d heat_buoyancy and d loss / d drag_per_s (finite differences of the float32 forward, h = 1e-2)
    against central differences of the FP64 oracle's loss (h = 1e-3): of the same sign and within 10% (measured
    1.1% for heat_buoyancy and 6.9% for drag, whose small effect on the loss shows the float32 run's drift from
    FP64 over 12 substeps the most)."""
    import torch

    recipe, source, target, fit, _, _, _ = case
    grads = fit.scalar_gradients(torch.from_numpy(source.astype(np.float32)), torch.from_numpy(target.astype(np.float32)))
    for name, got in grads.items():
        value = getattr(recipe.forces, name)
        up = dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, **{name: value + FD_H}))
        down = dataclasses.replace(recipe, forces=dataclasses.replace(recipe.forces, **{name: value - FD_H}))
        want = (oracle_loss(up, source, target)[0] - oracle_loss(down, source, target)[0]) / (2 * FD_H)
        print(f"{name}: float32 fd {got:.6e}, fp64 fd {want:.6e}")
        assert got * want > 0 and abs(got - want) <= 1e-1 * abs(want), name
