"""Buoyancy and drag (mirrors chadmv/plume src/plume/sim/forces.py:13-48)."""

import math

from plume_b200 import _native as N


def apply_buoyancy(grid, gravity: float, heat_buoyancy: float, smoke_weight: float, ambient_k: float,
                   dt: float) -> None:
    """v += gravity * (heat_buoyancy * (T - ambient) / ambient - smoke_weight * smoke) * dt at the y-faces."""
    N.call("plume_buoyancy", grid.info, N.ptr(grid.v.data), N.ptr(grid.smoke.data), N.ptr(grid.temperature.data),
           gravity, heat_buoyancy, smoke_weight, ambient_k, dt, N.stream())


def apply_drag(grid, wind_mps, drag_per_s: float, dt: float) -> None:
    """Relaxes every face velocity toward the wind by exp(-drag_per_s * dt); nothing when drag is 0."""
    if drag_per_s == 0.0:
        return
    keep = math.exp(-drag_per_s * dt)
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_drag", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), N.f3(wind_mps), keep, N.stream())
