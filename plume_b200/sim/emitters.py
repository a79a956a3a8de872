"""Emitters (mirrors chadmv/plume src/plume/sim/emitters.py:23-153).

`emitter_params` packs the recipe's emitters into C structs (each with its own noise stream, its index);
`emit` applies every emitter active at `time_s` to smoke, temperature and the three face velocities in one
launch. Emitters travel as kernel arguments, so no device array is needed.
"""

from plume_b200 import _native as N
from plume_b200._native import PlumeEmitter as EmitterParams

SPHERE = 0
BOX = 1
BLEND_REFERENCE_S = 1.0 / 80.0


def emitter_params(emitters, device: str = "cuda:0"):
    params = (EmitterParams * len(emitters))()
    for index, s in enumerate(emitters):
        p = params[index]
        p.shape = SPHERE if s.shape == "sphere" else BOX
        p.center_m = N.f3(s.center_m)
        p.radius_m = s.radius_m
        p.half_size_m = N.f3(size / 2 for size in s.size_m)
        p.edge_softness = s.edge_softness
        p.start_s = s.start_s
        p.end_s = s.end_s
        p.smoke_per_s = s.smoke_per_s
        p.temperature_k = s.temperature_k
        p.velocity_mps = N.f3(s.velocity_mps)
        p.outward = 1 if s.velocity_mode == "outward" else 0
        p.noise_scale_m = s.noise.scale_m
        p.noise_strength = s.noise.strength
        p.stream = index
    return params


def emit(grid, emitters, seed: int, time_s: float, dt: float) -> None:
    """Applies every emitter active at `time_s` for one step of length `dt`."""
    N.call("plume_emit", grid.info, N.ptr(grid.smoke.data), N.ptr(grid.temperature.data), N.ptr(grid.u.data),
           N.ptr(grid.v.data), N.ptr(grid.w.data), emitters, len(emitters), seed, time_s, dt, N.stream())
