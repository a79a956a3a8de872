"""One simulation substep (mirrors chadmv/plume src/plume/sim/stepper.py:17-60).

The operator order is the reference's: emit, buoyancy, confinement, turbulence, drag, advect velocity,
project, advect smoke (holding its total), advect temperature, dissipate. The whole substep is one library
call (plume_step), which enqueues every kernel on the current stream without a host synchronisation; the
fields' data/next buffers are swapped here afterwards, as the reference's AdvectedField.swap does.
"""

import ctypes
import math

import torch

from plume_b200 import _native as N
from plume_b200.sim.conserve import SmokeBudget
from plume_b200.sim.emitters import emitter_params
from plume_b200.sim.multigrid import Multigrid
from plume_b200.sim.pressure import GaussSeidel
from plume_b200.sim.pressure_solver import make_pressure_solve
from plume_b200.sim.vorticity import VorticityConfinement


class Stepper:
    """Advances a grid one step at a time under a recipe's emitters, forces and dissipation."""

    def __init__(self, grid, recipe):
        self.grid = grid
        self.recipe = recipe
        self.emitters = emitter_params(recipe.emitter, grid.device)
        self.pressure_solve = make_pressure_solve(grid, recipe.solver)
        self.smoke_budget = SmokeBudget(grid)
        self.confinement = VorticityConfinement(grid) if recipe.forces.vorticity_confinement > 0 else None
        # MacCormack's clamp ranges, kept between its forward pass and its correction
        self.advect_scratch = torch.empty(N.lib().plume_advect_scratch_floats(grid.info), dtype=torch.float32,
                                          device=grid.device)

    def _params(self, time_s: float, dt: float) -> N.PlumeStepParams:
        recipe, grid = self.recipe, self.grid
        forces, turbulence, dissipation = recipe.forces, recipe.forces.turbulence, recipe.dissipation
        p = N.PlumeStepParams()
        p.time_s, p.dt, p.dt_over_cell = time_s, dt, dt / grid.info.cell_m
        p.seed = recipe.seed
        p.emitters = ctypes.cast(self.emitters, ctypes.POINTER(N.PlumeEmitter))
        p.emitter_count = len(self.emitters)
        p.gravity, p.heat_buoyancy = forces.gravity_mps2, forces.heat_buoyancy
        p.smoke_weight, p.ambient_k = forces.smoke_weight, recipe.domain.ambient_k
        p.confinement = forces.vorticity_confinement if self.confinement is not None else 0.0
        if turbulence.strength_mps2 != 0.0:
            p.turbulence_scale_m = turbulence.scale_m
            p.turbulence_strength = turbulence.strength_mps2
            p.turbulence_pattern_time = time_s * turbulence.speed_mps / turbulence.scale_m
        if forces.drag_per_s != 0.0:
            p.apply_drag = 1
            p.wind = N.f3(forces.wind_mps)
            p.drag_keep = math.exp(-forces.drag_per_s * dt)
        solve = self.pressure_solve
        if isinstance(solve, Multigrid):
            p.solver, p.solver_iterations, p.multigrid_sweeps = 0, solve.cycles, solve.sweeps
        elif isinstance(solve, GaussSeidel):
            p.solver, p.solver_iterations = 1, solve.iterations
        else:
            raise TypeError(f"plume_step runs Multigrid or GaussSeidel solves, not {type(solve).__name__}")
        if dissipation.smoke_per_s != 0.0 or dissipation.cooling_per_s != 0.0:
            p.apply_dissipation = 1
            p.smoke_keep = math.exp(-dissipation.smoke_per_s * dt)
            p.heat_keep = math.exp(-dissipation.cooling_per_s * dt)
        return p

    def _state(self) -> N.PlumeStepState:
        grid = self.grid
        s = N.PlumeStepState()
        s.info = grid.info
        for name in ("u", "v", "w", "smoke", "temperature"):
            field = getattr(grid, name)
            setattr(s, name, N.PlumeField(N.field_ptr(field.data).value, N.field_ptr(field.hat).value,
                                          N.field_ptr(field.next).value))
        s.pressure, s.divergence = N.ptr(grid.pressure).value, N.ptr(grid.divergence).value
        if self.confinement is not None:
            s.curl = (ctypes.c_void_p * 3)(*[N.ptr(t).value for t in self.confinement._curl])
            s.push = (ctypes.c_void_p * 3)(*[N.ptr(t).value for t in self.confinement._push])
        s.sums = self.smoke_budget.sums.data_ptr()
        s.advect_scratch = N.ptr(self.advect_scratch).value
        s.factor = N.ptr(self.smoke_budget.factor).value
        if isinstance(self.pressure_solve, Multigrid):
            levels = self.pressure_solve.native_levels(grid)
        else:
            levels = (N.PlumeLevel * 1)()
            levels[0].info = grid.info
            levels[0].q, levels[0].rhs = N.ptr(grid.pressure).value, N.ptr(grid.divergence).value
            levels[0].residual = N.ptr(self.pressure_solve.second_array(grid)).value
        self._levels = levels
        s.levels = ctypes.cast(levels, ctypes.POINTER(N.PlumeLevel))
        s.level_count = len(levels)
        s.storage = N.storage_of(grid.smoke.data)
        return s

    def step(self, time_s: float, dt: float) -> None:
        """Advances from `time_s` to `time_s + dt`."""
        N.call("plume_step", self._state(), self._params(time_s, dt), N.stream())
        for field in (*self.grid.velocity_fields(), self.grid.smoke, self.grid.temperature):
            field.swap()
