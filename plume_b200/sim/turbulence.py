"""Curl-noise turbulence (mirrors chadmv/plume src/plume/sim/turbulence.py:59-67)."""

from plume_b200 import _native as N

TURBULENCE_STREAM = 1 << 24


def apply_turbulence(grid, seed: int, scale_m: float, strength_mps2: float, speed_mps: float, time_s: float,
                     dt: float) -> None:
    """Adds one step of the curl-noise push at time `time_s`; nothing when strength is 0."""
    if strength_mps2 == 0.0:
        return
    pattern_time = time_s * speed_mps / scale_m
    u, v, w = (f.data for f in grid.velocity_fields())
    N.call("plume_turbulence", grid.info, N.ptr(u), N.ptr(v), N.ptr(w), seed, scale_m, strength_mps2, pattern_time,
           dt, N.stream())
