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


class FlowFit:
    """The thickness loss's gradient through the whole step: with respect to the source field, and to the
    buoyancy and drag scalars (forces.heat_buoyancy, forces.drag_per_s), whose effect reaches the smoke only
    through the velocity. No reference counterpart.

    Model: SourceFit's (a source field added to the smoke at the start of every substep in its window, then the
    recipe's step); any smoke weight, vorticity confinement and turbulence. The forward run
    steps operator by operator (stepper.py:28-44, the two-pass advection) and keeps the full state (velocity,
    smoke, temperature and the pressure the next solve starts from) every `checkpoint_every` substeps. The
    backward pass walks the segments from the last, recomputes each segment's substeps keeping what the
    adjoint needs, then applies each substep's adjoint in reverse:
      dissipation; the smoke budget (uniform terms from its totals); MacCormack of smoke and temperature, with
      respect to the fields and to the advecting velocity (both traces' endpoints and midpoints); the
      projection, whose adjoint is the projection itself (walls zeroed, divergence, solve, gradient: the
      operator is symmetric), solved by `adjoint_cycles` V-cycles (the recipe's count by default) or refined
      to `solve_tol`; MacCormack of the velocity by itself (as field and as advector); drag (d/d drag_per_s);
      turbulence, whose push does not depend on the velocity (its adjoint passes the derivative through);
      vorticity confinement (through the push, the normalised spin gradient, the spin and the curl; d/d
      vorticity_confinement); buoyancy (to temperature and smoke, d/d heat_buoyancy); the emitter's blends; the
      source add (d/d source).
    The forward solve runs the recipe's V-cycles from the previous substep's pressure. The adjoint's solve
    starts, with `warm_start`, from the adjoint pressure of the substep after it (the one solved just before
    in the backward walk), else from zero. Either way the gradient is that of the exact projection, to within
    the residual the solves leave.

    Tape: a substep's record is 12 face arrays (15 with confinement) and 5 cell arrays. The forward pass of loss_and_grad keeps the
    records of the last segments whole while they fit `tape_bytes` (by default half the device memory free when
    the gradient is asked for), and the backward pass recomputes only the segments it did not keep. The forward
    is deterministic, so a kept record and a recomputed one are the same floats, and the budget changes the
    time, not the gradient."""

    def __init__(self, recipe, source_shape, corner, substeps: int, device: str = "cuda:0", window=(0.0, math.inf),
                 checkpoint_every: int = 8, adjoint_cycles: int | None = None, solve_tol: float | None = None,
                 warm_start: bool = True, tape_bytes: int | None = None):
        from plume_b200.sim.multigrid import Multigrid

        f = recipe.forces
        if recipe.solver.pressure_solver != "multigrid":
            raise ValueError("FlowFit needs the multigrid pressure solve")
        self.recipe, self.derived = recipe, derive(recipe)
        self.device = device
        self.source_shape, self.corner = tuple(source_shape), tuple(corner)
        self.substeps, self.window, self.every = substeps, window, checkpoint_every
        if adjoint_cycles is None:
            adjoint_cycles = recipe.solver.multigrid_cycles
        self.adjoint_cycles, self.solve_tol, self.warm_start = adjoint_cycles, solve_tol, warm_start
        self.tape_bytes = tape_bytes
        self.view = sheet_domain_view(recipe, self.derived)
        self.view_params = domain_view_params(self.view)
        self.emitters = emitter_params(recipe.emitter, device)
        d = recipe.domain
        self.grid = make_grid(self.derived, d.cell_m, d.faces, d.ambient_k, device)
        self.multigrid = Multigrid(self.grid, recipe.solver.multigrid_cycles, recipe.solver.multigrid_sweeps)
        self.adjoint_grid = make_grid(self.derived, d.cell_m, d.faces, d.ambient_k, device)
        self.adjoint_multigrid = Multigrid(self.adjoint_grid, adjoint_cycles, recipe.solver.multigrid_sweeps)
        info = self.grid.info
        self.sums = torch.empty(N.lib().plume_smoke_scratch_doubles(info), dtype=torch.float64, device=device)
        self.factor = torch.empty(1, dtype=torch.float32, device=device)
        self.partial = torch.empty(1024, dtype=torch.float64, device=device)
        self.coeffs = torch.empty(4, dtype=torch.float64, device=device)
        self.confined = f.vorticity_confinement > 0.0  # the step applies confinement only for a positive strength
        if self.confined:
            cells = self.grid.smoke.data.shape
            self.curl = [torch.empty(cells, dtype=torch.float32, device=device) for _ in range(3)]
            self.push = [torch.empty(cells, dtype=torch.float32, device=device) for _ in range(3)]
            self.confinement_scratch = torch.empty(N.lib().plume_confinement_adjoint_scratch_floats(info),
                                                   dtype=torch.float32, device=device)

    # ---- forward -----------------------------------------------------------------------------------------
    def _active(self, time_s: float) -> bool:
        return self.window[0] <= time_s < self.window[1]

    def _keeps(self, dt):
        diss = self.recipe.dissipation
        if diss.smoke_per_s == 0.0 and diss.cooling_per_s == 0.0:
            return None
        return math.exp(-diss.smoke_per_s * dt), math.exp(-diss.cooling_per_s * dt)

    def _load(self, state):
        g = self.grid
        for name, value in zip(("u", "v", "w", "smoke", "temperature"), state[:5]):
            getattr(g, name).data.copy_(value)
        g.pressure.copy_(state[5])

    def _state(self):
        g = self.grid
        return tuple(getattr(g, n).data.clone() for n in ("u", "v", "w", "smoke", "temperature")) + (
            g.pressure.clone(),)

    def _substep(self, n: int, source: torch.Tensor, record: bool = False):
        """Substep n on the work grid; with `record`, returns what its adjoint needs."""
        g, recipe, info = self.grid, self.recipe, self.grid.info
        dt, f, ambient = self.derived.dt_s, recipe.forces, recipe.domain.ambient_k
        time_s = n * dt
        if self._active(time_s):
            N.call("plume_add_source", N.ptr(g.smoke.data), N.shape3(g.smoke.data), N.ptr(source),
                   N.c_int3(*self.source_shape), N.c_int3(*self.corner), dt, N.stream())
        N.call("plume_emit", info, N.ptr(g.smoke.data), N.ptr(g.temperature.data), N.ptr(g.u.data), N.ptr(g.v.data),
               N.ptr(g.w.data), self.emitters, len(self.emitters), recipe.seed, time_s, dt, N.stream())
        N.call("plume_buoyancy", info, N.ptr(g.v.data), N.ptr(g.smoke.data), N.ptr(g.temperature.data),
               f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, ambient, dt, N.stream())
        rec = {}
        if self.confined:
            if record:
                rec["velocity_before_confinement"] = tuple(x.data.clone() for x in g.velocity_fields())
            N.call("plume_confinement", info, N.ptr(g.u.data), N.ptr(g.v.data), N.ptr(g.w.data), N.ptrs(*self.curl),
                   N.ptrs(*self.push), f.vorticity_confinement, dt, 1, N.stream())
        turbulence = f.turbulence
        if turbulence.strength_mps2 != 0.0:
            N.call("plume_turbulence", info, N.ptr(g.u.data), N.ptr(g.v.data), N.ptr(g.w.data), recipe.seed,
                   turbulence.scale_m, turbulence.strength_mps2, time_s * turbulence.speed_mps / turbulence.scale_m,
                   dt, N.stream())
        if record:
            rec["velocity_before_drag"] = tuple(x.data.clone() for x in g.velocity_fields())
        if f.drag_per_s != 0.0:
            N.call("plume_drag", info, N.ptr(g.u.data), N.ptr(g.v.data), N.ptr(g.w.data), N.f3(f.wind_mps),
                   math.exp(-f.drag_per_s * dt), N.stream())
        fields = g.velocity_fields()
        velocity = tuple(x.data for x in fields)
        if record:
            rec["velocity_advected"] = tuple(x.clone() for x in velocity)
        for x in fields:
            N.call("plume_advect_maccormack", info, N.shape3(x.data), N.ptr(x.data), N.ptr(x.hat), N.ptr(x.next),
                   *(N.ptr(y) for y in velocity), dt / info.cell_m, N.f3(x.offset), 0.0, 0, N.stream())
        if record:
            rec["velocity_hats"] = tuple(x.hat.clone() for x in fields)
        for x in fields:
            x.swap()
        u, v, w = (x.data for x in fields)
        N.call("plume_project_begin", info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(g.divergence), N.stream())
        self.multigrid(g)
        N.call("plume_subtract_gradient", info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(g.pressure), N.stream())
        if record:
            rec["velocity_projected"] = (u.clone(), v.clone(), w.clone())
            rec["smoke"], rec["temperature"] = g.smoke.data.clone(), g.temperature.data.clone()
        for field, outside in ((g.smoke, 0.0), (g.temperature, ambient)):
            N.call("plume_advect_maccormack", info, N.shape3(field.data), N.ptr(field.data), N.ptr(field.hat),
                   N.ptr(field.next), N.ptr(u), N.ptr(v), N.ptr(w), dt / info.cell_m, N.f3(CENTER), outside, 1,
                   N.stream())
        totals = torch.empty(3, dtype=torch.float64, device=self.device)
        if record:
            rec["smoke_hat"], rec["temperature_hat"] = g.smoke.hat.clone(), g.temperature.hat.clone()
            rec["smoke_next"] = g.smoke.next.clone()
            rec["totals"] = totals
        N.call("plume_smoke_budget", info, N.ptr(g.smoke.data), N.ptr(g.smoke.hat), N.ptr(g.smoke.next),
               N.ptr(self.sums, torch.float64), N.ptr(self.factor), N.ptr(totals, torch.float64), N.stream())
        g.smoke.swap()
        g.temperature.swap()
        keeps = self._keeps(dt)
        if keeps is not None:
            N.call("plume_dissipate", info, N.ptr(g.smoke.data), N.ptr(g.temperature.data), keeps[0], keeps[1],
                   ambient, N.stream())
        return rec

    def forward(self, source: torch.Tensor, taped_from: int | None = None):
        """The run from rest with the source; returns the checkpoints (one full state every checkpoint_every
        substeps) and leaves the final state in the work grid. With `taped_from`, also returns the records of
        substeps taped_from.. (a dict by substep)."""
        g = self.grid
        for x in (*g.velocity_fields(), g.smoke):
            x.data.zero_()
        g.temperature.data.fill_(self.recipe.domain.ambient_k)
        g.pressure.zero_()
        checkpoints, records = [], {}
        for n in range(self.substeps):
            if n % self.every == 0:
                checkpoints.append(self._state())
            taped = taped_from is not None and n >= taped_from
            rec = self._substep(n, source, record=taped)
            if taped:
                records[n] = rec
        return (checkpoints, records) if taped_from is not None else checkpoints

    def record_bytes(self) -> int:
        """Device bytes of one substep's record."""
        g = self.grid
        faces = sum(x.data.numel() for x in g.velocity_fields())
        return 4 * ((5 if self.confined else 4) * faces + 5 * g.smoke.data.numel()) + 8 * 3

    def _taped_from(self) -> int:
        """The first substep whose record the forward keeps: whole segments from the end, within the budget."""
        budget = self.tape_bytes
        if budget is None:
            free, _ = torch.cuda.mem_get_info(torch.device(self.device))
            budget = free // 2
        keep = int(budget // self.record_bytes())
        first = self.substeps - keep
        if first <= 0:
            return 0
        return min(self.substeps, -(-first // self.every) * self.every)

    def _thickness(self, target):
        g = self.grid
        height, width = self.view.height_px, self.view.width_px
        thickness = torch.empty((height, width), dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        a_smoke = torch.zeros_like(g.smoke.data)
        N.call("plume_thickness_adjoint", g.info, self.view_params, self.recipe.render.opacity_per_density,
               N.ptr(g.smoke.data), N.ptr(target), height, width, N.ptr(thickness), N.ptr(loss, torch.float64),
               N.ptr(a_smoke), N.stream())
        return float(loss.item()), thickness, a_smoke

    def loss(self, source: torch.Tensor, target: torch.Tensor) -> float:
        source = source.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        self.forward(source)
        return self._thickness(target)[0]

    def with_forces(self, **forces) -> "FlowFit":
        recipe = dataclasses.replace(self.recipe, forces=dataclasses.replace(self.recipe.forces, **forces))
        return FlowFit(recipe, self.source_shape, self.corner, self.substeps, self.device, self.window, self.every,
                       self.adjoint_cycles, self.solve_tol, self.warm_start, self.tape_bytes)

    # ---- backward ----------------------------------------------------------------------------------------
    def _project_adjoint(self, a_vel):
        """a_vel <- P a_vel: the projection, its solve adjoint_cycles V-cycles (or refined) from the last
        adjoint pressure (warm_start) or from zero."""
        from plume_b200.sim.pressure import project, project_refined

        adj = self.adjoint_grid
        for x, a in zip(adj.velocity_fields(), a_vel):
            x.data.copy_(a)
        if not self.warm_start:
            adj.pressure.zero_()
        if self.solve_tol is None:
            project(adj, self.adjoint_multigrid)
        else:
            project_refined(adj, self.adjoint_multigrid, rel_tol=self.solve_tol)
        for x, a in zip(adj.velocity_fields(), a_vel):
            a.copy_(x.data)

    def _substep_adjoint(self, n, rec, a_smoke, a_heat, a_vel, grads, grad_source):
        """Reverse of substep n: (a_smoke, a_heat, a_vel) of the state after it -> of the state before it."""
        g, recipe, info = self.grid, self.recipe, self.grid.info
        dt, f, ambient = self.derived.dt_s, recipe.forces, recipe.domain.ambient_k
        dtc = dt / info.cell_m
        keeps = self._keeps(dt) or (1.0, 1.0)
        time_s = n * dt
        # smoke budget and dissipation
        a_next = torch.empty_like(a_smoke)
        a_smoke_in = torch.empty_like(a_smoke)
        a_smoke_hat = torch.empty_like(a_smoke)
        N.call("plume_budget_adjoint", info, N.ptr(rec["smoke_next"]), N.ptr(rec["totals"], torch.float64),
               keeps[0], N.ptr(a_smoke), N.ptr(a_next), N.ptr(a_smoke_in), N.ptr(a_smoke_hat),
               N.ptr(self.partial, torch.float64), N.ptr(self.coeffs, torch.float64), N.stream())
        a_heat_next = a_heat * keeps[1]
        a_heat_in = torch.zeros_like(a_heat)
        a_heat_hat = torch.zeros_like(a_heat)
        vp = rec["velocity_projected"]
        # scalar MacCormack with the velocity's derivative; a_vel is the projected velocity's
        for data, hat, a_out, a_in, a_hat, outside in (
                (rec["smoke"], rec["smoke_hat"], a_next, a_smoke_in, a_smoke_hat, 0.0),
                (rec["temperature"], rec["temperature_hat"], a_heat_next, a_heat_in, a_heat_hat, ambient)):
            N.call("plume_maccormack_adjoint", info, N.shape3(data), N.f3(CENTER), N.ptr(data), N.ptr(hat),
                   *(N.ptr(x) for x in vp), N.ptr(a_out), N.ptr(a_in), N.ptr(a_hat), *(N.ptr(x) for x in a_vel),
                   dtc, outside, 1, N.stream())
        # the projection
        self._project_adjoint(a_vel)
        # velocity MacCormack, the velocity as field and as advector
        vd = rec["velocity_advected"]
        a_vd = tuple(torch.zeros_like(x) for x in a_vel)
        for component, (x, hat, a_out) in enumerate(zip(vd, rec["velocity_hats"], a_vel)):
            a_hat = torch.zeros_like(x)
            N.call("plume_maccormack_adjoint", info, N.shape3(x), N.f3(g.velocity_fields()[component].offset),
                   N.ptr(x), N.ptr(hat), *(N.ptr(y) for y in vd), N.ptr(a_out), N.ptr(a_vd[component]),
                   N.ptr(a_hat), *(N.ptr(y) for y in a_vd), dtc, 0.0, 0, N.stream())
        # drag, buoyancy, the emitter's blends, the source
        if f.drag_per_s != 0.0:
            N.call("plume_drag_adjoint", info, *(N.ptr(x) for x in a_vd),
                   *(N.ptr(x) for x in rec["velocity_before_drag"]), N.f3(f.wind_mps), math.exp(-f.drag_per_s * dt),
                   dt, N.ptr(grads[1:2], torch.float64), N.stream())
        # turbulence's push does not depend on the velocity: its adjoint is the identity
        if self.confined:
            N.call("plume_confinement_adjoint", info, *(N.ptr(x) for x in rec["velocity_before_confinement"]),
                   *(N.ptr(x) for x in a_vd), f.vorticity_confinement, dt, N.ptr(self.confinement_scratch),
                   N.ptr(grads[2:3], torch.float64), N.stream())
        N.call("plume_buoyancy_adjoint", info, N.ptr(a_vd[1]), N.ptr(rec["smoke"]), N.ptr(rec["temperature"]),
               N.ptr(a_smoke_in), N.ptr(a_heat_in), f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, ambient, dt,
               N.ptr(grads[0:1], torch.float64), N.stream())
        N.call("plume_emit_adjoint", info, N.ptr(a_heat_in), *(N.ptr(x) for x in a_vd), self.emitters,
               len(self.emitters), recipe.seed, time_s, dt, N.stream())
        if self._active(time_s):
            N.call("plume_source_grad", N.ptr(a_smoke_in), N.shape3(a_smoke_in), N.ptr(grad_source),
                   N.c_int3(*self.source_shape), N.c_int3(*self.corner), dt, N.stream())
        return a_smoke_in, a_heat_in, list(a_vd)

    def loss_and_grad(self, source: torch.Tensor, target: torch.Tensor):
        """(loss, d loss / d source, {"heat_buoyancy": ..., "drag_per_s": ...[, "vorticity_confinement": ...]},
        final thickness); the confinement strength's derivative when the recipe applies confinement."""
        source = source.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        taped_from = self._taped_from()
        checkpoints, taped = self.forward(source, taped_from)
        loss, thickness, a_smoke = self._thickness(target)
        g = self.grid
        self.adjoint_grid.pressure.zero_()
        a_heat = torch.zeros_like(g.temperature.data)
        a_vel = [torch.zeros_like(x.data) for x in g.velocity_fields()]
        grads = torch.zeros(3, dtype=torch.float64, device=self.device)
        grad_source = torch.zeros(self.source_shape, dtype=torch.float32, device=self.device)
        for segment in reversed(range(len(checkpoints))):
            first = segment * self.every
            last = min(first + self.every, self.substeps)
            if first >= taped_from:
                records = [taped.pop(n) for n in range(first, last)]
            else:
                self._load(checkpoints[segment])
                records = [self._substep(n, source, record=True) for n in range(first, last)]
            for n in reversed(range(first, last)):
                a_smoke, a_heat, a_vel = self._substep_adjoint(n, records[n - first], a_smoke, a_heat, a_vel, grads,
                                                               grad_source)
            del records
        hb, drag, eps = (float(x) for x in grads.cpu())
        scalars = {"heat_buoyancy": hb, "drag_per_s": drag}
        if self.confined:
            scalars["vorticity_confinement"] = eps
        return loss, grad_source, scalars, thickness
