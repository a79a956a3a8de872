"""The fused MacCormack passes (plume_maccormack_velocity, plume_maccormack_scalars) against the FP32 oracle's
advect_maccormack (the reference's advect.py:59-68: semi-Lagrangian forward, backward, clamped correction) on
the same seeded fields, called through the C ABI.

The fused passes blend with fused multiply-adds, about an ulp from the reference's a*(1-t) + b*t, so each
result is held to the per-operator tolerance of 1e-5 as a relative error of the field: the largest difference
over the field's largest magnitude (a value that cancels to near zero carries the rounding of its operands, so
an element-by-element ratio would measure that cancellation, not the operator). Two time steps:
dt = 1/96 s keeps every trace within a cell (served from the staged planes in shared memory); dt = 8/96 s
sends traces several cells (served from global memory). Grid shapes cover one tile, partial tiles, several
x segments per column and the v/w end rows."""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from plume_b200 import _native as N
from plume_b200.workloads import operator_fields
from support import ALL_CLOSED, OPEN, cuda_grid, host, load_state, oracle_grid

pytestmark = pytest.mark.gpu

OP_RTOL = 1e-5
TOTAL_RTOL = 1e-6  # the smoke budget's totals (line sums split at the x segments)
CASES = [((32, 48, 32), OPEN), ((32, 48, 32), ALL_CLOSED), ((15, 17, 13), OPEN), ((3, 5, 2), ALL_CLOSED),
         ((40, 70, 100), OPEN), ((33, 16, 31), ALL_CLOSED)]
IDS = ["32x48x32-open", "32x48x32-closed", "15x17x13-open", "3x5x2-closed", "40x70x100-open", "33x16x31-closed"]
DTS = [1.0 / 96.0, 8.0 / 96.0]


def pair(cells, faces, seed=11, cell_m=1.0 / 64.0, ambient_k=1.0):
    o = oracle_grid(cells, cell_m, faces, ambient_k)
    c = cuda_grid(cells, cell_m, faces, ambient_k)
    load_state(o, c, operator_fields(cells, seed, ambient_k))
    return o, c


def check(actual, expected, what):
    scale = float(np.abs(expected).max()) or 1.0
    err = float(np.abs(np.asarray(actual, np.float64) - expected).max()) / scale
    assert err < OP_RTOL, f"{what}: {err:.3g} of the field's largest magnitude {scale:.3g}"


@pytest.mark.parametrize("dt", DTS, ids=["dt1", "dt8"])
@pytest.mark.parametrize("cells,faces", CASES, ids=IDS)
def test_fused_velocity_advection_matches_the_oracle(cuda_device, cells, faces, dt):
    o, c = pair(cells, faces)
    velocity = tuple(f.data for f in o.velocity_fields())
    for name in ("u", "v", "w"):
        O.advect_maccormack(getattr(o, name), velocity, o, dt)
    out = [torch.full_like(getattr(c, name).data, float("nan")) for name in ("u", "v", "w")]
    N.call("plume_maccormack_velocity", c.info, *(N.ptr(getattr(c, n).data) for n in ("u", "v", "w")),
           *(N.ptr(t) for t in out), dt / c.info.cell_m, N.stream())
    torch.cuda.synchronize()
    for name, tensor in zip(("u", "v", "w"), out):
        check(host(tensor), getattr(o, name).next, name)


def scalars(c, dt, outside=(0.0, 1.0), uses_outside=1):
    smoke_next = torch.full_like(c.smoke.data, float("nan"))
    heat_next = torch.full_like(c.temperature.data, float("nan"))
    scratch = torch.empty(N.lib().plume_maccormack_scratch_floats(c.info), dtype=torch.float32, device="cuda:0")
    sums = torch.empty(N.lib().plume_smoke_scratch_doubles(c.info), dtype=torch.float64, device="cuda:0")
    totals = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    N.call("plume_maccormack_scalars", c.info, *(N.ptr(f.data) for f in c.velocity_fields()), N.ptr(c.smoke.data),
           N.ptr(c.temperature.data), N.ptr(smoke_next), N.ptr(heat_next), dt / c.info.cell_m, outside[0],
           outside[1], uses_outside, N.ptr(scratch), N.ptr(sums, torch.float64), N.ptr(totals, torch.float64),
           N.stream())
    torch.cuda.synchronize()
    return host(smoke_next), host(heat_next), totals.cpu().numpy()


@pytest.mark.parametrize("dt", DTS, ids=["dt1", "dt8"])
@pytest.mark.parametrize("cells,faces", CASES, ids=IDS)
def test_fused_smoke_and_temperature_advection_match_the_oracle(cuda_device, cells, faces, dt):
    o, c = pair(cells, faces)
    velocity = tuple(f.data for f in o.velocity_fields())
    O.advect_maccormack(o.smoke, velocity, o, dt)
    O.advect_maccormack(o.temperature, velocity, o, dt)
    smoke, heat, totals = scalars(c, dt)
    check(smoke, o.smoke.next, "smoke")
    check(heat, o.temperature.next, "temperature")
    expected = [O.total(a, o.precision) for a in (o.smoke.data, o.smoke.hat, o.smoke.next)]
    for name, got, want in zip(("before", "semi-Lagrangian", "MacCormack"), totals, expected):
        assert abs(got - want) <= TOTAL_RTOL * abs(want), f"{name} total {got!r} vs {want!r}"


def test_fused_advection_is_deterministic(cuda_device):
    _, c = pair((40, 70, 100), OPEN)
    first = scalars(c, 8.0 / 96.0)
    second = scalars(c, 8.0 / 96.0)
    for a, b in zip(first, second):
        assert np.array_equal(a, b)
