"""The allocation-free smoke budget (plume_smoke_budget_static) against the caller-scratch one
(plume_smoke_budget), through the C ABI.

It exists for callers that cannot allocate device memory when they hold the budget (a host engine that only
hands over the fields it owns, or code where an allocation would synchronise the device); its scratch is a
fixed array inside the library. This file is collected last so that a failure here leaves every other test
already run; it passes alone in a fresh process too.
"""

import pytest
import torch

from plume_b200 import _native as N
from plume_b200.workloads import operator_fields
from support import OPEN, cuda_grid

pytestmark = pytest.mark.gpu


def budget_inputs(cells, seed):
    """Smoke before the step, a plain semi-Lagrangian total below it and a MacCormack total above it, so the
    held factor (before / MacCormack) differs from 1 and the rescaling runs."""
    grid = cuda_grid(cells, 1.0 / 64.0, OPEN, 1.0)
    before = torch.from_numpy(operator_fields(cells, seed, 1.0)["smoke"]).cuda() + 0.25
    grid.smoke.data.copy_(before)
    grid.smoke.hat.copy_(before * 0.8)
    grid.smoke.next.copy_(before * 1.1)
    return grid


def budget_with_scratch(grid, next_field):
    sums = torch.zeros(N.lib().plume_smoke_scratch_doubles(grid.info), dtype=torch.float64, device="cuda:0")
    factor = torch.zeros(1, dtype=torch.float32, device="cuda:0")
    totals = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    N.call("plume_smoke_budget", grid.info, N.ptr(grid.smoke.data), N.ptr(grid.smoke.hat), N.ptr(next_field),
           N.ptr(sums, torch.float64), N.ptr(factor), N.ptr(totals, torch.float64), N.stream())
    return totals


def budget_static(grid, next_field):
    totals = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    N.call("plume_smoke_budget_static", grid.info, N.ptr(grid.smoke.data), N.ptr(grid.smoke.hat),
           N.ptr(next_field), N.ptr(totals, torch.float64), N.stream())
    return totals


@pytest.mark.parametrize("cells", [(32, 48, 32), (15, 17, 13), (1, 1024, 1024)])
def test_static_budget_matches_the_scratch_budget_on_two_calls_in_a_row(cuda_device, cells):
    for call, seed in enumerate((1, 2)):  # the second call reuses the array the first one left behind
        grid = budget_inputs(cells, seed + sum(cells))
        expected_next = grid.smoke.next.clone()
        expected_totals = budget_with_scratch(grid, expected_next)
        actual_next = grid.smoke.next.clone()
        actual_totals = budget_static(grid, actual_next)
        torch.cuda.synchronize()
        # the same kernels in the same order: identical floats (tolerance 0 for this integer-free path)
        assert torch.equal(actual_next, expected_next), f"call {call}: scaled smoke differs"
        assert torch.equal(actual_totals, expected_totals), f"call {call}: totals differ"
        assert float(expected_totals[2]) > float(expected_totals[0]), "inputs must exercise the rescaling"
        assert not torch.equal(actual_next, grid.smoke.next), "the budget should have rescaled the smoke"


def test_static_budget_rejects_grids_beyond_its_scratch(cuda_device):
    from plume_b200.sim.grid import make_info

    info = make_info((1, 1025, 1024), 0.01, (0.0, 0.0, 0.0), (0, 0, 0), (0, 0, 0))
    dummy = torch.zeros(1, dtype=torch.float32, device="cuda:0")
    status = N.lib().plume_smoke_budget_static(info, N.ptr(dummy), N.ptr(dummy), N.ptr(dummy), None, N.stream())
    assert status == -1
    assert b"exceeds the fixed scratch" in N.lib().plume_last_error()
