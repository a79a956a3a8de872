"""The pressure solve's launch strategies (tiled sweeps, per-colour launches, one-block and cluster coarse
solves, CUDA-graph replay) all give the oracle's pressure bit for bit."""

import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from support import ALL_CLOSED, OPEN, assert_same, blob, cuda_grid, host, load_state, oracle_grid

pytestmark = pytest.mark.gpu

# odd sizes: several tiles, coarse levels with overhanging cells (non-uniform stencil)
CASES = [((19, 24, 17), OPEN), ((40, 36, 70), ALL_CLOSED), ((38, 48, 38), OPEN), ((5, 33, 66), OPEN),
         ((70, 9, 7), ALL_CLOSED), ((32, 48, 32), OPEN)]
IDS = ["19x24x17-open", "40x36x70-closed", "38x48x38-open", "5x33x66-open", "70x9x7-closed", "32x48x32-open"]


@pytest.fixture
def tuning(cuda_device):
    from plume_b200.sim.multigrid import solver_tuning, tune_solver

    saved = solver_tuning()
    yield saved
    tune_solver(saved)


def seeded_pair(cells, faces):
    o, c = oracle_grid(cells, 0.05, faces), cuda_grid(cells, 0.05, faces)
    rng = np.random.default_rng(sum(cells))
    fields = {"u": rng.uniform(-1, 1, (cells[0] + 1, cells[1], cells[2])),
              "v": rng.uniform(-1, 1, (cells[0], cells[1] + 1, cells[2])),
              "w": rng.uniform(-1, 1, (cells[0], cells[1], cells[2] + 1)),
              "pressure": 0.01 * blob(cells, [n / 3 for n in cells], 3.0)}
    load_state(o, c, {k: v.astype(np.float32) for k, v in fields.items()})
    return o, c


@pytest.mark.parametrize("cells,faces", CASES, ids=IDS)
@pytest.mark.parametrize("tiled_min", [1, 1 << 40])
@pytest.mark.parametrize("bottom_max", [0, 2048, 8192])  # uniform levels of <= 2048 cells use register stencils
def test_multigrid_strategies_match_the_oracle(tuning, cells, faces, tiled_min, bottom_max):
    from plume_b200.sim.multigrid import Multigrid, tune_solver
    from plume_b200.sim.pressure import project

    tune_solver(dataclasses.replace(tuning, tiled_min_cells=tiled_min, bottom_max_cells=bottom_max))
    for sweeps in (2, 3):
        o, c = seeded_pair(cells, faces)
        O.project(o, O.Multigrid(o, 2, sweeps))
        project(c, Multigrid(c, 2, sweeps))
        assert_same(host(c.pressure), o.pressure, f"pressure, {sweeps} sweeps")
        for name in ("u", "v", "w"):
            assert_same(host(getattr(c, name).data), getattr(o, name).data, name)


@pytest.mark.parametrize("cells,faces", CASES[:3], ids=IDS[:3])
@pytest.mark.parametrize("tiled_min", [1, 1 << 40])
def test_gauss_seidel_strategies_match_the_oracle(tuning, cells, faces, tiled_min):
    from plume_b200.sim.multigrid import tune_solver
    from plume_b200.sim.pressure import GaussSeidel, project

    tune_solver(dataclasses.replace(tuning, tiled_min_cells=tiled_min))
    o, c = seeded_pair(cells, faces)
    O.project(o, O.GaussSeidel(7))
    project(c, GaussSeidel(7))
    assert_same(host(c.pressure), o.pressure, "pressure after 7 sweeps")


@pytest.mark.parametrize("bottom_kind", [0, 1])
@pytest.mark.parametrize("graphs", [0, 1])
def test_every_strategy_gives_the_same_pressure(tuning, bottom_kind, graphs):
    from plume_b200 import _native as N
    from plume_b200.sim.multigrid import Multigrid, tune_solver
    from plume_b200.sim.pressure import project

    cells, faces = (38, 48, 38), OPEN
    o, _ = seeded_pair(cells, faces)
    O.project(o, O.Multigrid(o, 3, 2))
    try:
        N.call("plume_use_graphs", graphs)
        for tiled_min, bottom_max in ((1, 0), (1, 8192), (20000, 2000), (1 << 40, 8192)):
            tune_solver(dataclasses.replace(tuning, tiled_min_cells=tiled_min, bottom_max_cells=bottom_max,
                                            bottom_kind=bottom_kind))
            _, c = seeded_pair(cells, faces)
            project(c, Multigrid(c, 3, 2))
            assert_same(host(c.pressure), o.pressure, f"tiled_min {tiled_min}, bottom {bottom_max}/{bottom_kind}")
    finally:
        N.call("plume_use_graphs", 1)


def test_tuning_rejects_bad_values(tuning):
    from plume_b200.sim.multigrid import tune_solver

    for bad in (dict(tiled_min_cells=0), dict(bottom_max_cells=-1), dict(bottom_kind=2)):
        with pytest.raises(RuntimeError):
            tune_solver(dataclasses.replace(tuning, **bad))


def test_the_autotuner_picks_the_fastest_candidate_and_restores_the_pressure(tuning):
    import torch

    from plume_b200.sim.autotune import autotune_solver
    from plume_b200.sim.multigrid import solver_tuning
    from plume_b200.sim.pressure import compute_divergence

    _, c = seeded_pair((38, 48, 38), OPEN)
    compute_divergence(c)
    before = c.pressure.clone()
    result = autotune_solver(c, 2, 2, repeats=2)
    assert len(result.ms_per_solve) == 5 and all(ms > 0.0 for ms in result.ms_per_solve.values())
    assert result.best == min(result.ms_per_solve, key=result.ms_per_solve.get)
    assert solver_tuning() == result.best
    assert torch.equal(c.pressure, before)


@pytest.fixture
def split_threshold(cuda_device):
    from plume_b200 import _native as N

    default = N.lib().plume_split_min_cells()
    N.call("plume_tune_split", 1)  # every top level runs split, whatever its size
    yield
    N.call("plume_tune_split", default)


@pytest.mark.parametrize("cells,faces", CASES + [((24, 20, 33), OPEN), ((31, 17, 9), ALL_CLOSED)],
                         ids=IDS + ["24x20x33-open", "31x17x9-closed"])
def test_colour_split_top_level_gives_the_same_pressure(split_threshold, cells, faces):
    """The top level swept in colour-split storage (red and black cells in separate arrays, odd rows padded)
    gives plume_multigrid's pressure bit for bit, with a warm start and 2 or 3 sweeps."""
    import torch

    from plume_b200 import _native as N
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence

    for sweeps in (2, 3):
        _, a = seeded_pair(cells, faces)
        _, b = seeded_pair(cells, faces)
        compute_divergence(a)
        compute_divergence(b)
        ma, mb = Multigrid(a, 2, sweeps), Multigrid(b, 2, sweeps)
        ma(a)
        scratch = torch.empty(N.lib().plume_split_scratch_floats(b.info), dtype=torch.float32, device="cuda:0")
        levels = mb.native_levels(b)
        N.call("plume_multigrid_split", levels, len(mb.levels), 2, sweeps, N.ptr(scratch), N.stream())
        torch.cuda.synchronize()
        assert_same(host(b.pressure), host(a.pressure), f"pressure, {sweeps} sweeps")
