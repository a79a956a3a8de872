"""Choosing the pressure solve a recipe asks for (mirrors chadmv/plume src/plume/sim/pressure_solver.py:9-13)."""

from plume_b200.sim.multigrid import Multigrid
from plume_b200.sim.pressure import GaussSeidel


def make_pressure_solve(grid, solver):
    if solver.pressure_solver == "gauss_seidel":
        return GaussSeidel(solver.pressure_iterations)
    return Multigrid(grid, solver.multigrid_cycles, solver.multigrid_sweeps)
