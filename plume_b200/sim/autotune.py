"""Choosing the pressure solve's strategy by measurement (no reference counterpart). Every strategy gives the
same pressure bit for bit (the solver tests check it), so the choice is speed alone: each candidate solves
the grid's current problem a few times under CUDA events and the fastest is set for the process. The grid's
pressure is restored afterwards."""

import dataclasses

import torch

from plume_b200.sim.multigrid import Multigrid, SolverTuning, solver_tuning, tune_solver

# one-block bottom from the first level of at most 512, 2048 or 8192 cells; tiled sweeps on the largest levels
# (at least 2^20 cells) or never; the 8-CTA cluster bottom at 2048 cells
DEFAULT_CANDIDATES = ((1 << 40, 2048, 0), (1 << 40, 512, 0), (1 << 40, 8192, 0), (1 << 20, 2048, 0),
                      (1 << 40, 2048, 1))


@dataclasses.dataclass(frozen=True)
class TuningResult:
    best: SolverTuning
    ms_per_solve: dict  # SolverTuning -> milliseconds per solve


def autotune_solver(grid, cycles: int, sweeps: int, candidates=DEFAULT_CANDIDATES, repeats: int = 5,
                    apply: bool = True) -> TuningResult:
    """Times `cycles` V-cycles of `sweeps` sweeps on the grid's current divergence under each candidate
    (tiled_min_cells, bottom_max_cells, bottom_kind) and returns the fastest; with `apply` it stays set."""
    start_tuning = solver_tuning()
    saved = grid.pressure.clone()
    multigrid = Multigrid(grid, cycles, sweeps)
    times = {}
    try:
        for tiled, bottom, kind in candidates:
            tuning = dataclasses.replace(start_tuning, tiled_min_cells=tiled, bottom_max_cells=bottom,
                                         bottom_kind=kind)
            tune_solver(tuning)
            grid.pressure.copy_(saved)
            multigrid(grid)  # warm-up: the graph capture
            begin, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            begin.record()
            for _ in range(repeats):
                multigrid(grid)
            end.record()
            torch.cuda.synchronize()
            times[tuning] = begin.elapsed_time(end) / repeats
    finally:
        grid.pressure.copy_(saved)
        tune_solver(start_tuning)
    best = min(times, key=times.get)
    if apply:
        tune_solver(best)
    return TuningResult(best, times)
