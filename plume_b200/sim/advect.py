"""Clamped MacCormack advection (mirrors chadmv/plume src/plume/sim/advect.py:53-76).

One call enqueues the forward semi-Lagrangian pass (into `field.hat`) and the correction, which evaluates
the backward pass in place and clamps to the eight values the forward sample blended (into `field.next`).
"""

import ctypes

from plume_b200 import _native as N


def advect_semi_lagrangian(field, velocity, grid, dt: float) -> None:
    """Plain semi-Lagrangian advection into `field.next`."""
    u, v, w = velocity
    N.call("plume_advect_semi_lagrangian", grid.info, N.shape3(field.data), N.ptr(field.data), N.ptr(field.next),
           N.ptr(u), N.ptr(v), N.ptr(w), dt / grid.info.cell_m, N.f3(field.offset),
           field.outside, field.uses_outside, N.stream())


def advect_maccormack(field, velocity, grid, dt: float) -> None:
    """Clamped MacCormack advection of `field.data` into `field.next`."""
    u, v, w = velocity
    N.call("plume_advect_maccormack", grid.info, N.shape3(field.data), N.ptr(field.data), N.ptr(field.hat),
           N.ptr(field.next), N.ptr(u), N.ptr(v), N.ptr(w), dt / grid.info.cell_m,
           N.f3(field.offset), field.outside, field.uses_outside, N.stream())
