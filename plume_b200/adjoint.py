"""Derivatives of a rendered thickness loss with respect to a smoke source field: the hand-written adjoint of
the step's smoke path and of the thickness march (libplume_b200's plume_smoke_adjoint and
plume_thickness_adjoint), behind a torch.autograd.Function. The reference has no derivatives; this is the
differentiable form of its step for fitting a source to a target image.

Model: a source field (nonnegative smoke per second on a box of cells, its corner at `corner`) is added to the
smoke at the start of every substep in its active window, then the step runs as usual (Stepper.step). With
forces.smoke_weight = 0 the velocity does not depend on the smoke, so the loss depends on the source only
through the smoke path -- the source add, MacCormack advection of the smoke by the step's velocity, the smoke
budget and dissipation -- and the march. The forward run records each substep's velocity and a smoke
checkpoint every `checkpoint_every` substeps; the backward pass walks the segments from the last, recomputing
each segment's smoke states from its checkpoint and then applying the adjoint substep by substep.
"""

import dataclasses
import math

import torch

from plume_b200 import _native as N
from plume_b200.recipe.derived import derive
from plume_b200.render.camera import sheet_domain_view
from plume_b200.render.frame_renderer import domain_view_params
from plume_b200.sim.emitters import emitter_params
from plume_b200.sim.grid import CENTER, make_grid
from plume_b200.sim.stepper import Stepper


class SourceFit:
    """loss = sum over pixels (thickness of the final state - target)^2, and d loss / d source."""

    def __init__(self, recipe, source_shape, corner, substeps: int, device: str = "cuda:0", window=(0.0, math.inf),
                 checkpoint_every: int = 8, initial_state=None):
        if recipe.forces.smoke_weight != 0.0:
            raise ValueError("the source adjoint needs forces.smoke_weight = 0 (velocity independent of the smoke)")
        self.recipe, self.derived = recipe, derive(recipe)
        self.device = device
        self.source_shape, self.corner = tuple(source_shape), tuple(corner)
        self.substeps, self.window, self.every = substeps, window, checkpoint_every
        self.initial_state = initial_state
        self.view = sheet_domain_view(recipe, self.derived)
        self.view_params = domain_view_params(self.view)
        self.emitters = emitter_params(recipe.emitter, device)

    def _active(self, time_s: float) -> bool:
        return self.window[0] <= time_s < self.window[1]

    def _add(self, smoke, source, scale):
        N.call("plume_add_source", N.ptr(smoke), N.shape3(smoke), N.ptr(source), N.c_int3(*self.source_shape),
               N.c_int3(*self.corner), scale, N.stream())

    def forward(self, source: torch.Tensor):
        """Runs the recipe for `substeps` with the source; returns the final grid and the tape."""
        d = self.recipe.domain
        grid = make_grid(self.derived, d.cell_m, d.faces, d.ambient_k, self.device)
        if self.initial_state is not None:
            self.initial_state(grid)
        stepper = Stepper(grid, self.recipe)
        dt = self.derived.dt_s
        checkpoints, velocities = [], []
        for n in range(self.substeps):
            if n % self.every == 0:
                checkpoints.append(grid.smoke.data.clone())
            if self._active(n * dt):
                self._add(grid.smoke.data, source, dt)
            stepper.step(n * dt, dt)
            velocities.append(tuple(f.data.clone() for f in grid.velocity_fields()))
        return grid, (checkpoints, velocities)

    def loss(self, source: torch.Tensor, target: torch.Tensor) -> float:
        """The loss alone (a forward run and the march)."""
        source = source.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        grid, _ = self.forward(source)
        height, width = self.view.height_px, self.view.width_px
        thickness = torch.empty((height, width), dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        scratch = torch.zeros_like(grid.smoke.data)
        N.call("plume_thickness_adjoint", grid.info, self.view_params, self.recipe.render.opacity_per_density,
               N.ptr(grid.smoke.data), N.ptr(target), height, width, N.ptr(thickness), N.ptr(loss, torch.float64),
               N.ptr(scratch), N.stream())
        return float(loss.item())

    def with_forces(self, **forces) -> "SourceFit":
        """The same fit with some of recipe.forces changed (e.g. heat_buoyancy, drag_per_s)."""
        recipe = dataclasses.replace(self.recipe, forces=dataclasses.replace(self.recipe.forces, **forces))
        return SourceFit(recipe, self.source_shape, self.corner, self.substeps, self.device, self.window, self.every,
                         self.initial_state)

    def scalar_gradients(self, source: torch.Tensor, target: torch.Tensor, names=("heat_buoyancy", "drag_per_s"),
                         h: float = 1e-2) -> dict:
        """d loss / d each named recipe.forces scalar, by central differences of the forward loss (two forward
        runs per scalar, step h). These scalars move the velocity, whose adjoint is not built: the source
        field's gradient is the adjoint's (loss_and_grad), the scalars' are finite differences."""
        grads = {}
        for name in names:
            value = getattr(self.recipe.forces, name)
            up = self.with_forces(**{name: value + h}).loss(source, target)
            down = self.with_forces(**{name: value - h}).loss(source, target)
            grads[name] = (up - down) / (2.0 * h)
        return grads

    def _smoke_substep(self, smoke, n, source, scratch):
        """Recomputes substep n's smoke path from `smoke` (its start state); returns (data, hat, next_pre,
        totals, out)."""
        dt = self.derived.dt_s
        recipe, info = self.recipe, scratch["info"]
        data = smoke.clone()
        if self._active(n * dt):
            self._add(data, source, dt)
        dummy_t, (du, dv, dw) = scratch["temperature"], scratch["velocity"]
        N.call("plume_emit", info, N.ptr(data), N.ptr(dummy_t), N.ptr(du), N.ptr(dv), N.ptr(dw), self.emitters,
               len(self.emitters), recipe.seed, n * dt, dt, N.stream())
        u, v, w = scratch["velocities"][n]
        hat, next_pre = torch.empty_like(data), torch.empty_like(data)
        N.call("plume_advect_maccormack", info, N.shape3(data), N.ptr(data), N.ptr(hat), N.ptr(next_pre), N.ptr(u),
               N.ptr(v), N.ptr(w), dt / info.cell_m, N.f3(CENTER), 0.0, 1, N.stream())
        totals = torch.empty(3, dtype=torch.float64, device=self.device)
        out = next_pre.clone()
        N.call("plume_smoke_budget", info, N.ptr(data), N.ptr(hat), N.ptr(out), N.ptr(scratch["sums"], torch.float64),
               N.ptr(scratch["factor"]), N.ptr(totals, torch.float64), N.stream())
        keep = scratch["keep"]
        if keep != 1.0:
            N.call("plume_dissipate", info, N.ptr(out), N.ptr(dummy_t), keep, 1.0, recipe.domain.ambient_k, N.stream())
        return data, hat, next_pre, totals, out

    def loss_and_grad(self, source: torch.Tensor, target: torch.Tensor):
        """(loss, d loss / d source, final thickness image); target is the (height, width) thickness."""
        source = source.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        grid, (checkpoints, velocities) = self.forward(source)
        info = grid.info
        height, width = self.view.height_px, self.view.width_px
        thickness = torch.empty((height, width), dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        a_smoke = torch.zeros_like(grid.smoke.data)
        N.call("plume_thickness_adjoint", info, self.view_params, self.recipe.render.opacity_per_density,
               N.ptr(grid.smoke.data), N.ptr(target), height, width, N.ptr(thickness), N.ptr(loss, torch.float64),
               N.ptr(a_smoke), N.stream())
        grad = torch.zeros(self.source_shape, dtype=torch.float32, device=self.device)
        dt = self.derived.dt_s
        dissipation = self.recipe.dissipation
        scratch = {"info": info, "velocities": velocities,
                   "temperature": torch.zeros_like(grid.smoke.data),  # emit's other outputs, discarded
                   "velocity": tuple(torch.zeros_like(f.data) for f in grid.velocity_fields()),
                   "sums": torch.empty(N.lib().plume_smoke_scratch_doubles(info), dtype=torch.float64,
                                       device=self.device),
                   "factor": torch.empty(1, dtype=torch.float32, device=self.device),
                   "keep": math.exp(-dissipation.smoke_per_s * dt) if (dissipation.smoke_per_s != 0.0 or
                                                                       dissipation.cooling_per_s != 0.0) else 1.0}
        a_next, a_hat, a_data = (torch.empty_like(a_smoke) for _ in range(3))
        partial = torch.empty(1024, dtype=torch.float64, device=self.device)
        coeffs = torch.empty(4, dtype=torch.float64, device=self.device)
        for segment in reversed(range(len(checkpoints))):
            first = segment * self.every
            last = min(first + self.every, self.substeps)
            states, smoke = [], checkpoints[segment]
            for n in range(first, last):
                data, hat, next_pre, totals, out = self._smoke_substep(smoke, n, source, scratch)
                states.append((data, hat, next_pre, totals))
                smoke = out
            for n in reversed(range(first, last)):
                data, hat, next_pre, totals = states[n - first]
                u, v, w = velocities[n]
                N.call("plume_smoke_adjoint", info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(data), N.ptr(hat),
                       N.ptr(next_pre), N.ptr(totals, torch.float64), dt / info.cell_m, scratch["keep"],
                       N.ptr(a_smoke), N.ptr(a_next), N.ptr(a_hat), N.ptr(a_data), N.ptr(partial, torch.float64),
                       N.ptr(coeffs, torch.float64), N.stream())
                if self._active(n * dt):
                    N.call("plume_source_grad", N.ptr(a_data), N.shape3(a_data), N.ptr(grad),
                           N.c_int3(*self.source_shape), N.c_int3(*self.corner), dt, N.stream())
                a_smoke, a_data = a_data, a_smoke
        return float(loss.item()), grad, thickness


class ThicknessLoss(torch.autograd.Function):
    """loss = SourceFit(...).loss for a source tensor, with its hand-written gradient."""

    @staticmethod
    def forward(ctx, source, fit: SourceFit, target):
        loss, grad, _ = fit.loss_and_grad(source.detach(), target)
        ctx.save_for_backward(grad)
        return torch.tensor(loss, dtype=torch.float64, device=source.device)

    @staticmethod
    def backward(ctx, grad_output):
        (grad,) = ctx.saved_tensors
        return (grad_output.to(grad.dtype) * grad).to(grad.dtype), None, None
