"""Holding clamped MacCormack's smoke total within the scheme's own bounds (mirrors chadmv/plume
src/plume/sim/conserve.py:33-52).

After each smoke advection the MacCormack total is held between the plain semi-Lagrangian total and the
total before the step by scaling the whole field by one factor. Here the totals, the factor and the scaling
all stay on the device: no host synchronisation per substep.
"""

import torch

from plume_b200 import _native as N


def held_total(before: float, semi_lagrangian: float, maccormack: float) -> float:
    return max(semi_lagrangian, min(maccormack, before))


class SmokeBudget:
    """Scratch for one grid's smoke totals and its last factor (a device float)."""

    def __init__(self, grid):
        self.sums = torch.zeros(N.lib().plume_smoke_scratch_doubles(grid.info), dtype=torch.float64,
                                device=grid.device)
        self.factor = torch.ones(1, dtype=torch.float32, device=grid.device)
        self.totals = torch.zeros(3, dtype=torch.float64, device=grid.device)

    @property
    def last_factor(self) -> float:
        return float(self.factor.item())

    def hold(self, grid) -> None:
        """Call after advecting smoke and before swapping: rescales grid.smoke.next into its bounds."""
        s = grid.smoke
        N.call("plume_smoke_budget", grid.info, N.ptr(s.data), N.ptr(s.hat), N.ptr(s.next),
               N.ptr(self.sums, torch.float64), N.ptr(self.factor), N.ptr(self.totals, torch.float64), N.stream())
