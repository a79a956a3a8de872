"""Geometric multigrid for the pressure solve (mirrors chadmv/plume src/plume/sim/multigrid.py:24-147).

Cell-centred V-cycles with averaging restriction and trilinear prolongation. Levels halve each axis
(rounding up) until the shortest axis is at most 2 cells or there are 8 levels; a coarse level's overhanging
last cell is weighted by the share inside the domain (`fill_hi`). The whole V-cycle runs in one library call.
"""

import math
from dataclasses import dataclass

import torch

from plume_b200 import _native as N
from plume_b200.sim.grid import GridInfo, make_info

MIN_LEVEL_CELLS = 2
MAX_LEVELS = 8
COARSEST_SWEEPS = 20
COARSEST_SWEEPS_PER_CELL = 4
COARSEST_RELAXATION = 1.5
SMOOTHING_RELAXATION = 1.0


@dataclass(frozen=True)
class SolverTuning:
    """The library's pressure-solve strategy (results do not depend on it): levels of at least
    `tiled_min_cells` cells sweep in shared-memory tiles, one launch per sweep; smaller ones one colour per
    launch; the first level of at most `bottom_max_cells` cells and all coarser ones run in one launch
    (`bottom_kind` 0 one block, 1 an 8-CTA cluster)."""

    tiled_min_cells: int
    bottom_max_cells: int
    bottom_kind: int


def solver_tuning() -> SolverTuning:
    values = (N.ctypes.c_longlong(), N.ctypes.c_longlong(), N.ctypes.c_int32())
    N.call("plume_solver_tuning", *(N.ctypes.byref(v) for v in values))
    return SolverTuning(*(int(v.value) for v in values))


def tune_solver(tuning: SolverTuning) -> None:
    N.call("plume_tune_solver", tuning.tiled_min_cells, tuning.bottom_max_cells, tuning.bottom_kind)


@dataclass
class Level:
    info: GridInfo
    cells: tuple
    q: torch.Tensor
    rhs: torch.Tensor
    residual: torch.Tensor


@dataclass(frozen=True)
class Refinement:
    """What Multigrid.refine did: the correction cycles run; ||rhs - A q|| / ||rhs|| (double precision, 2-norms)
    of the iterate before the first correction and after each one; and that ratio for the float pressure
    left in grid.pressure (the iterate rounded to float)."""

    corrections: int
    ratios: tuple
    float_ratio: float

    @property
    def ratio(self) -> float:
        return self.ratios[-1]


def coarse_cells(cells):
    return tuple((n + 1) // 2 for n in cells)


def coarse_geometry(top_cells, cells, level: int):
    """(fill_hi, ghost_gap) of a level `level` steps down: the share of its last cell inside the domain on each
    axis, and the distance in its cells to the pressure-0 ghost beyond an open face."""
    scale = 2.0 ** level
    return tuple(top / scale - (n - 1) for top, n in zip(top_cells, cells)), 0.5 / scale


class Multigrid:
    """`cycles` V-cycles per solve, with `sweeps` smoothing sweeps before and after each correction."""

    def __init__(self, grid, cycles: int, sweeps: int):
        self.cycles = cycles
        self.sweeps = sweeps
        self.device = grid.device
        self.levels = self._build_levels(grid)
        self._native_levels = None
        self._refine = None

    def _build_levels(self, grid):
        levels = [Level(grid.info, grid.cells, grid.pressure, grid.divergence,
                        torch.zeros(grid.cells, dtype=torch.float32, device=grid.device))]
        while min(levels[-1].cells) > MIN_LEVEL_CELLS and len(levels) < MAX_LEVELS:
            above = levels[-1]
            cells = coarse_cells(above.cells)
            fill, gap = coarse_geometry(grid.cells, cells, len(levels))
            info = make_info(cells, above.info.cell_m * 2.0, tuple(above.info.origin_m), tuple(above.info.open_lo),
                             tuple(above.info.open_hi), fill, gap)
            levels.append(Level(info, cells, *(torch.zeros(cells, dtype=torch.float32, device=self.device)
                                               for _ in range(3))))
        return levels

    def native_levels(self, grid):
        """The levels as the C structs the library reads (the top level aliases the grid's arrays)."""
        self.levels[0].q = grid.pressure
        self.levels[0].rhs = grid.divergence
        array = (N.PlumeLevel * len(self.levels))()
        for slot, level in zip(array, self.levels):
            slot.info = level.info
            slot.q = N.ptr(level.q).value
            slot.rhs = N.ptr(level.rhs).value
            slot.residual = N.ptr(level.residual).value
        self._native_levels = array
        return array

    def __call__(self, grid) -> None:
        levels = self.native_levels(grid)
        N.call("plume_multigrid", levels, len(self.levels), self.cycles, self.sweeps, N.stream())

    def refine(self, grid, rel_tol: float = 1e-7, max_corrections: int = 40, compensated: bool = True) -> Refinement:
        """Solves to a relative residual by defect correction (no reference counterpart; the reference runs a
        fixed number of V-cycles). Each correction evaluates r = divergence - A pressure in double, solves
        A e = r with one float V-cycle from e = 0 whose coarsest level is swept in double, and adds e to the
        pressure. With `compensated` the iterate is grid.pressure + a second float array of its rounding error
        (two-sum), so it can go below the float pressure's own rounding floor (about 4e-7 on the seeded
        operator fields); grid.pressure always holds the iterate rounded to float. Stops at
        ||r|| / ||divergence|| <= rel_tol, after max_corrections, or when a correction improves the ratio by
        less than 5%."""
        self.native_levels(grid)
        top = self.levels[0]
        if self._refine is None or self._refine["e"].shape != grid.pressure.shape:
            cells = grid.cells
            blocks = N.lib().plume_norm_scratch_doubles(N.ctypes.byref(top.info))
            self._refine = {name: torch.zeros(cells, dtype=torch.float32, device=self.device) for name in ("e", "r", "ping")}
            self._refine["scratch"] = torch.empty(blocks, dtype=torch.float64, device=self.device)
            self._refine["norms"] = torch.zeros(2, dtype=torch.float64, device=self.device)
            self._refine["lo"] = torch.zeros(cells, dtype=torch.float32, device=self.device)
        arrays = self._refine
        arrays["lo"].zero_()
        lo = N.ptr(arrays["lo"]) if compensated else None
        levels = (N.PlumeLevel * len(self.levels))()
        for index, (slot, level) in enumerate(zip(levels, self.levels)):
            slot.info = level.info
            if index == 0:
                slot.q, slot.rhs, slot.residual = (N.ptr(arrays[name]).value for name in ("e", "r", "ping"))
            else:
                slot.q, slot.rhs, slot.residual = (N.ptr(t).value for t in (level.q, level.rhs, level.residual))

        def measure(low) -> float:
            N.call("plume_residual_f64", top.info, N.ptr(grid.pressure), low, N.ptr(grid.divergence),
                   N.ptr(arrays["r"]), N.ptr(arrays["scratch"], torch.float64), N.ptr(arrays["norms"], torch.float64),
                   N.stream())
            rr, bb = (float(x) for x in arrays["norms"].cpu())
            return 0.0 if bb == 0.0 else math.sqrt(rr / bb)

        ratios = [measure(lo)]
        corrections = 0
        while ratios[-1] > rel_tol and corrections < max_corrections:
            N.call("plume_multigrid_correct", levels, len(self.levels), self.sweeps, N.ptr(grid.pressure), lo,
                   N.stream())
            corrections += 1
            ratios.append(measure(lo))
            if ratios[-1] > 0.95 * ratios[-2]:
                break
        float_ratio = measure(None) if compensated else ratios[-1]
        return Refinement(corrections, tuple(ratios), float_ratio)

    def residual(self, level_index: int = 0) -> torch.Tensor:
        """Fills and returns one level's residual rhs - A q (multigrid.py:36-43)."""
        level = self.levels[level_index]
        N.call("plume_residual", level.info, N.ptr(level.q), N.ptr(level.rhs), N.ptr(level.residual), N.stream())
        return level.residual
