"""Pressure projection (mirrors chadmv/plume src/plume/sim/pressure.py:17-162).

Solves laplacian(q) = divergence(u) for a scaled pressure q, then subtracts gradient(q) from the face
velocities. Closed faces are walls; open faces see q = 0 just outside. The solve is pluggable: GaussSeidel
here, Multigrid in plume_b200.sim.multigrid.
"""

from typing import Protocol

import torch

from plume_b200 import _native as N

RELAXATION = 1.5


class PressureSolve(Protocol):
    def __call__(self, grid) -> None:
        """Improves grid.pressure toward the solution of laplacian(q) = grid.divergence."""


class GaussSeidel:
    """A fixed number of red-black Gauss-Seidel sweeps with over-relaxation."""

    def __init__(self, iterations: int):
        self.iterations = iterations
        self.scratch = None

    def second_array(self, grid) -> torch.Tensor:
        """The sweeps' second pressure array (each sweep reads one and writes the other)."""
        if self.scratch is None or self.scratch.shape != grid.pressure.shape:
            self.scratch = torch.empty_like(grid.pressure)
        return self.scratch

    def __call__(self, grid) -> None:
        red_black_sweeps(grid.pressure, grid.divergence, grid.info, grid.cells, grid.device, self.iterations,
                         RELAXATION, self.second_array(grid))


def red_black_sweeps(q, rhs, info, cells, device, sweeps: int, relaxation: float, scratch=None) -> None:
    """`sweeps` red-black sweeps (colour 0 then 1) of laplacian(q) = rhs on the grid `info` describes."""
    scratch = torch.empty_like(q) if scratch is None else scratch
    N.call("plume_red_black_sweeps", info, N.ptr(q), N.ptr(scratch), N.ptr(rhs), sweeps, relaxation, N.stream())


def project(grid, solve) -> None:
    """Makes the face velocities divergence-free (to the solver's accuracy) and walls impermeable."""
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_project_begin", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(grid.divergence), N.stream())
    solve(grid)
    N.call("plume_subtract_gradient", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(grid.pressure), N.stream())


def project_refined(grid, multigrid, rel_tol: float = 1e-6, max_corrections: int = 40):
    """project() with the pressure solved to a relative residual by multigrid.refine (defect correction; no
    reference counterpart). Returns the Refinement."""
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_project_begin", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(grid.divergence), N.stream())
    refinement = multigrid.refine(grid, rel_tol, max_corrections)
    N.call("plume_subtract_gradient", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(grid.pressure), N.stream())
    return refinement


def compute_divergence(grid):
    """Fills and returns grid.divergence from the current face velocities."""
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_divergence", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(grid.divergence), N.stream())
    return grid.divergence
