"""Solving the pressure to a relative residual by defect correction (no reference counterpart): the double
residual and its norms against the FP64 oracle, the tolerance reached on the seeded operator fields, and the
refined float pressure against a converged FP64 oracle solve."""

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.workloads import operator_fields
from support import ALL_CLOSED, OPEN, cuda_grid, host, load_state, oracle_grid

pytestmark = pytest.mark.gpu


def seeded(cells, faces, precision="f32", seed=11):
    o = oracle_grid(cells, 1.0 / 64.0, faces, 1.0, precision)
    c = cuda_grid(cells, 1.0 / 64.0, faces, 1.0)
    fields = operator_fields(cells, seed, 1.0)
    fields["pressure"] = (0.01 * np.random.default_rng(seed).standard_normal(cells)).astype(np.float32)
    load_state(o, c, fields)
    return o, c


@pytest.mark.parametrize("cells,faces", [((24, 32, 20), OPEN), ((19, 24, 17), ALL_CLOSED)])
def test_double_residual_and_norms_match_the_fp64_oracle(cuda_device, cells, faces):
    import torch

    from plume_b200 import _native as N
    from plume_b200.sim.pressure import compute_divergence

    o, c = seeded(cells, faces, "f64")
    O.compute_divergence(o)
    compute_divergence(c)
    o.divergence[...] = host(c.divergence)  # the same float right-hand side on both sides
    expected = O.Multigrid(o, 1, 2).residual(o)
    residual = torch.empty_like(c.pressure)
    scratch = torch.empty(N.lib().plume_norm_scratch_doubles(N.ctypes.byref(c.info)), dtype=torch.float64,
                          device="cuda:0")
    norms = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    N.call("plume_residual_f64", c.info, N.ptr(c.pressure), None, N.ptr(c.divergence), N.ptr(residual),
           N.ptr(scratch, torch.float64), N.ptr(norms, torch.float64), N.stream())
    scale = np.abs(expected).max()
    assert np.abs(host(residual) - expected).max() <= 1e-6 * scale
    rr, bb = host(norms)
    assert abs(rr - np.sum(expected * expected)) <= 1e-9 * rr
    assert abs(bb - np.sum(host(c.divergence).astype(np.float64) ** 2)) <= 1e-12 * bb


@pytest.mark.parametrize("cells", [(64, 96, 64), (128, 192, 128)])
def test_refine_reaches_the_relative_residual(cuda_device, cells):
    """The seeded operator fields of the 128x192x128 correctness case (and half its size): the projection's
    pressure reaches a relative residual of 1e-6 in float alone and 1e-7 as a compensated float pair; the
    plain 4 V-cycles stop near 1e-4."""
    import torch

    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence

    c = cuda_grid(cells, 1.0 / 64.0, OPEN, 1.0)
    for name, values in operator_fields(cells, 11, 1.0).items():
        getattr(c, name).data.copy_(torch.from_numpy(values))
    compute_divergence(c)
    c.pressure.zero_()
    mg = Multigrid(c, 4, 2)
    plain = mg.refine(c, rel_tol=1.0).ratio  # measures only
    mg(c)
    after_cycles = mg.refine(c, rel_tol=1.0).ratio
    c.pressure.zero_()
    refined = mg.refine(c, rel_tol=1e-6, max_corrections=40, compensated=False)
    print(f"{cells}: start {plain:.3e}, after 4 V-cycles {after_cycles:.3e}; float: {refined.corrections} "
          f"corrections: {', '.join(f'{r:.2e}' for r in refined.ratios)}")
    assert refined.ratio <= 1e-6 and refined.corrections <= 20
    c.pressure.zero_()
    pair = mg.refine(c, rel_tol=1e-7, max_corrections=40)
    print(f"  compensated: {pair.corrections} corrections: {', '.join(f'{r:.2e}' for r in pair.ratios)}; "
          f"rounded to float {pair.float_ratio:.2e}")
    assert pair.ratio <= 1e-7 and pair.corrections <= 20
    assert pair.float_ratio <= 1e-6
    assert torch.isfinite(c.pressure).all()


def test_refined_pressure_matches_a_converged_fp64_solve(cuda_device):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence

    cells = (24, 32, 20)
    o, c = seeded(cells, OPEN, "f64")
    compute_divergence(c)
    o.divergence[...] = host(c.divergence)
    o.pressure[...] = 0.0
    c.pressure.zero_()
    O.Multigrid(o, 80, 2)(o)  # converged in double
    refined = Multigrid(c, 4, 2).refine(c, rel_tol=1e-7)
    assert refined.ratio <= 1e-6
    exact = o.pressure
    assert np.abs(host(c.pressure) - exact).max() <= 1e-5 * np.abs(exact).max()


@pytest.mark.parametrize("cells,faces", [((19, 24, 17), ALL_CLOSED), ((38, 48, 38), OPEN)],
                         ids=["19x24x17-closed", "38x48x38-open"])
def test_refine_on_closed_and_uneven_grids(cuda_device, cells, faces):
    """All walls closed (the pressure is defined up to a constant; the walls are closed first, as a projection
    does, so the divergence sums to zero) and levels with overhanging cells: the corrections shrink the
    residual far below the plain cycles' and the pressure stays finite."""
    import torch

    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import GaussSeidel, compute_divergence, project

    c = cuda_grid(cells, 1.0 / 64.0, faces, 1.0)
    for name, values in operator_fields(cells, 11, 1.0).items():
        getattr(c, name).data.copy_(torch.from_numpy(values))
    project(c, GaussSeidel(0))  # closes the walls
    compute_divergence(c)
    c.pressure.zero_()
    refined = Multigrid(c, 4, 2).refine(c, rel_tol=1e-7)
    print(f"{cells}: {refined.corrections} corrections: {', '.join(f'{r:.2e}' for r in refined.ratios)}")
    assert refined.ratio <= 1e-5 and refined.ratios[-1] < refined.ratios[0]
    assert torch.isfinite(c.pressure).all()
