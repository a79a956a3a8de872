"""Dissipation (mirrors chadmv/plume src/plume/sim/dissipate.py:18-24)."""

import math

from plume_b200 import _native as N


def dissipate(grid, smoke_per_s: float, cooling_per_s: float, ambient_k: float, dt: float) -> None:
    """Smoke fades by exp(-smoke_per_s dt); temperature relaxes toward ambient by exp(-cooling_per_s dt)."""
    if smoke_per_s == 0.0 and cooling_per_s == 0.0:
        return
    N.call("plume_dissipate", grid.info, N.ptr(grid.smoke.data), N.ptr(grid.temperature.data),
           math.exp(-smoke_per_s * dt), math.exp(-cooling_per_s * dt), ambient_k, N.stream())
