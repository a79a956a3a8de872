"""Deterministic totals of grid fields on the device (mirrors chadmv/plume src/plume/sim/reduce.py:28-38).

Each (j, k) line is summed along x in float32 in order; the lines are added in float64 in a fixed order
(blocks of 256 by a halving tree, then the block partials in order), so the same fields always give the same
totals.
"""

import torch

from plume_b200 import _native as N


class TripleSum:
    """Totals of three same-shaped fields; calling it copies three doubles to the host."""

    def __init__(self, shape, device: str):
        self.shape = tuple(shape)
        blocks = (shape[1] * shape[2] + 255) // 256
        self.sums = torch.zeros(3 * blocks, dtype=torch.float64, device=device)
        self.totals = torch.zeros(3, dtype=torch.float64, device=device)

    def device_totals(self, a, b, c) -> torch.Tensor:
        N.call("plume_triple_sum", N.c_int3(*self.shape), N.ptr(a), N.ptr(b), N.ptr(c),
               N.ptr(self.sums, torch.float64), N.ptr(self.totals, torch.float64), N.stream())
        return self.totals

    def __call__(self, a, b, c):
        totals = self.device_totals(a, b, c).cpu()
        return float(totals[0]), float(totals[1]), float(totals[2])
