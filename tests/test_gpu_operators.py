"""Operator parity: each CUDA operator, called through the C ABI, against the FP32 oracle on the same seeded
inputs. Operators without exp/pow must give identical floats; those with them (emitter blend, light volume,
ray march) must agree within the stated relative tolerance (exp/pow are evaluated in double on the device,
the C library's expf/powf in the oracle: at most about 1 ulp apart)."""

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.workloads import operator_fields
from support import ALL_CLOSED, FIELDS, OPEN, assert_same, cuda_grid, host, load_state, max_rel, oracle_grid

pytestmark = pytest.mark.gpu

EXP_POW_RTOL = 1e-5  # operators that call exp/pow
CASES = [((32, 48, 32), OPEN), ((32, 48, 32), ALL_CLOSED), ((15, 17, 13), OPEN), ((3, 5, 2), ALL_CLOSED)]
IDS = ["32x48x32-open", "32x48x32-closed", "15x17x13-open", "3x5x2-closed"]


def pair(cells, faces, cell_m=1.0 / 64.0, ambient_k=1.0, seed=11):
    """An oracle grid and a CUDA grid holding the same seeded operator-test fields."""
    o = oracle_grid(cells, cell_m, faces, ambient_k)
    c = cuda_grid(cells, cell_m, faces, ambient_k)
    load_state(o, c, operator_fields(cells, seed, ambient_k))
    return o, c


@pytest.mark.parametrize("cells,faces", CASES, ids=IDS)
@pytest.mark.parametrize("name", FIELDS)
def test_maccormack_matches_the_oracle(cuda_device, cells, faces, name):
    from plume_b200.sim.advect import advect_maccormack

    o, c = pair(cells, faces)
    dt = 1.0 / 96.0 * 8.0  # several cells per step: exercises traces across many cells
    O.advect_maccormack(getattr(o, name), tuple(f.data for f in o.velocity_fields()), o, dt)
    advect_maccormack(getattr(c, name), tuple(f.data for f in c.velocity_fields()), c, dt)
    assert_same(host(getattr(c, name).hat), getattr(o, name).hat, f"{name} hat")
    assert_same(host(getattr(c, name).next), getattr(o, name).next, f"{name} next")


@pytest.mark.parametrize("cells,faces", CASES[:3], ids=IDS[:3])
def test_semi_lagrangian_matches_the_oracle(cuda_device, cells, faces):
    from plume_b200.sim.advect import advect_semi_lagrangian

    o, c = pair(cells, faces)
    for name in FIELDS:
        O.advect_semi_lagrangian(getattr(o, name), tuple(f.data for f in o.velocity_fields()), o, 0.05)
        advect_semi_lagrangian(getattr(c, name), tuple(f.data for f in c.velocity_fields()), c, 0.05)
        assert_same(host(getattr(c, name).next), getattr(o, name).next, name)


def _emitter_recipe():
    from plume_b200.recipe.load import resolve_table

    table = {"seed": 5, "domain": {"size_m": [0.5, 0.75, 0.5], "cell_m": 1.0 / 64.0, "ambient_k": 1.0},
             "time": {"duration_s": 1.0},
             "emitter": [
                 {"name": "a", "center_m": [0.02, 0.2, -0.03], "radius_m": 0.12, "end_s": 1.0, "smoke_per_s": 3.0,
                  "temperature_k": 2.5, "velocity_mps": [0.1, 0.6, 0.0], "velocity_mode": "outward",
                  "edge_softness": 0.5, "noise": {"scale_m": 0.05, "strength": 0.8}},
                 {"name": "b", "shape": "box", "center_m": [-0.1, 0.1, 0.05], "size_m": [0.1, 0.08, 0.12],
                  "end_s": 1.0, "smoke_per_s": 2.0, "temperature_k": 3.0, "velocity_mps": [0.3, 0.2, -0.1],
                  "edge_softness": 0.3},
                 {"name": "late", "center_m": [0.0, 0.3, 0.0], "radius_m": 0.1, "start_s": 0.5, "end_s": 1.0,
                  "smoke_per_s": 9.0}]}
    return resolve_table(table, "emitters")


def test_emit_matches_the_oracle(cuda_device):
    from plume_b200.sim.emitters import emit, emitter_params

    recipe = _emitter_recipe()
    cells = (32, 48, 32)
    o, c = pair(cells, OPEN)
    for time_s in (0.0, 0.6):
        O.emit(o, O.emitter_params(recipe.emitter), recipe.seed, time_s, 0.0125)
        emit(c, emitter_params(recipe.emitter), recipe.seed, time_s, 0.0125)
    assert_same(host(c.smoke.data), o.smoke.data, "smoke")  # no exp/pow on the smoke path
    for name in ("temperature", "u", "v", "w"):
        assert max_rel(host(getattr(c, name).data), getattr(o, name).data, floor=1e-3) < EXP_POW_RTOL, name


# Spacings: a power of two, where the kernels multiply by the exact reciprocal of a spacing in place of dividing
# by it, and one that is not, where they divide; both must give the oracle's floats.
CELL_MS = [1.0 / 64.0, 0.1]
CELL_M_IDS = ["dx-1/64", "dx-0.1"]


@pytest.mark.parametrize("cell_m", CELL_MS, ids=CELL_M_IDS)
def test_forces_match_the_oracle(cuda_device, cell_m):
    from plume_b200.sim.forces import apply_buoyancy, apply_drag
    from plume_b200.sim.turbulence import apply_turbulence
    from plume_b200.sim.vorticity import VorticityConfinement

    for cells, faces in CASES:
        o, c = pair(cells, faces, cell_m=cell_m)
        O.apply_buoyancy(o, 1.0, 1.0, 0.05, 1.0, 0.02)
        apply_buoyancy(c, 1.0, 1.0, 0.05, 1.0, 0.02)
        assert_same(host(c.v.data), o.v.data, f"buoyancy {cells}")
        oc, cc = O.VorticityConfinement(o), VorticityConfinement(c)
        assert_same(host(cc.measure_curl(c)), oc.measure_curl(o), f"curl {cells}")
        oc.apply(o, 0.3, 0.02)
        cc.apply(c, 0.3, 0.02)
        assert_same(host(cc.push), oc.push, f"push {cells}")
        O.apply_turbulence(o, 3, 0.2, 0.5, 0.2, 0.37, 0.02)
        apply_turbulence(c, 3, 0.2, 0.5, 0.2, 0.37, 0.02)
        O.apply_drag(o, (0.2, 0.0, -0.1), 0.5, 0.02)
        apply_drag(c, (0.2, 0.0, -0.1), 0.5, 0.02)
        for name in ("u", "v", "w"):
            assert_same(host(getattr(c, name).data), getattr(o, name).data, f"{name} after forces {cells}")


@pytest.mark.parametrize("cell_m", CELL_MS, ids=CELL_M_IDS)
@pytest.mark.parametrize("cells,faces", CASES, ids=IDS)
def test_projection_matches_the_oracle(cuda_device, cells, faces, cell_m):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import GaussSeidel, compute_divergence, project

    for solver in ("gauss_seidel", "multigrid"):
        o, c = pair(cells, faces, cell_m=cell_m)
        if solver == "gauss_seidel":
            os_, cs = O.GaussSeidel(20), GaussSeidel(20)
        else:
            os_, cs = O.Multigrid(o, 2, 2), Multigrid(c, 2, 2)
            assert [lv.cells for lv in cs.levels] == [lv.cells for lv in os_.levels]
        O.project(o, os_)
        project(c, cs)
        assert_same(host(c.pressure), o.pressure, f"{solver} pressure")
        for name in ("u", "v", "w"):
            assert_same(host(getattr(c, name).data), getattr(o, name).data, f"{solver} {name}")
        assert_same(host(compute_divergence(c)), O.compute_divergence(o), f"{solver} divergence")


@pytest.mark.parametrize("cells", [(128, 256, 256), (129, 256, 255)], ids=["128x256x256", "129x256x255"])
def test_projection_on_a_level_beyond_l2_matches_the_oracle(cuda_device, cells):
    """Levels of at least 2^23 cells sweep two planes per thread: Gauss-Seidel sweeps and a V-cycle at that
    size (an odd plane count and an odd row length in the second case) give the oracle's floats."""
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import GaussSeidel, project

    assert cells[0] * cells[1] * cells[2] >= 1 << 23
    fields = operator_fields(cells, 11, 1.0)
    for solver in ("gauss_seidel", "multigrid"):
        o, c = oracle_grid(cells, 1.0 / 64.0, OPEN, 1.0), cuda_grid(cells, 1.0 / 64.0, OPEN, 1.0)
        load_state(o, c, fields)
        os_, cs = (O.GaussSeidel(3), GaussSeidel(3)) if solver == "gauss_seidel" else (O.Multigrid(o, 1, 2),
                                                                                     Multigrid(c, 1, 2))
        O.project(o, os_)
        project(c, cs)
        assert_same(host(c.pressure), o.pressure, f"{solver} pressure")


@pytest.mark.parametrize("cell_m", CELL_MS, ids=CELL_M_IDS)
def test_multigrid_residual_matches_the_oracle(cuda_device, cell_m):
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence

    o, c = pair((15, 17, 13), OPEN, cell_m=cell_m)
    O.compute_divergence(o)
    compute_divergence(c)
    om, cm = O.Multigrid(o, 1, 2), Multigrid(c, 1, 2)
    for _ in range(3):
        om(o)
        cm(c)
        assert_same(host(cm.residual()), om.residual(o), "residual")


def test_smoke_budget_dissipation_and_speed_match_the_oracle(cuda_device):
    from plume_b200.sim.advect import advect_maccormack
    from plume_b200.sim.conserve import SmokeBudget
    from plume_b200.sim.dissipate import dissipate
    from plume_b200.sim.reduce import TripleSum
    from plume_b200.sim.step_cap import StepCap

    o, c = pair((32, 48, 32), OPEN)
    O.advect_maccormack(o.smoke, tuple(f.data for f in o.velocity_fields()), o, 0.05)
    advect_maccormack(c.smoke, tuple(f.data for f in c.velocity_fields()), c, 0.05)
    sums = TripleSum(c.cells, c.device)(c.smoke.data, c.smoke.hat, c.smoke.next)
    p = o.precision
    assert sums == (O.total(o.smoke.data, p), O.total(o.smoke.hat, p), O.total(o.smoke.next, p))
    ob, cb = O.SmokeBudget(o), SmokeBudget(c)
    ob.hold(o)
    cb.hold(c)
    assert cb.last_factor == np.float32(ob.last_factor)
    assert_same(host(c.smoke.next), o.smoke.next, "held smoke")
    O.dissipate(o, 1.6, 1.0, 1.0, 0.0125)
    dissipate(c, 1.6, 1.0, 1.0, 0.0125)
    assert_same(host(c.smoke.data), o.smoke.data, "dissipated smoke")
    assert_same(host(c.temperature.data), o.temperature.data, "dissipated temperature")
    assert StepCap.grid_speed(c) == O.StepCap.grid_speed(o)


def test_triple_sum_matches_float64_numpy(cuda_device):
    import torch

    from plume_b200.sim.reduce import TripleSum

    rng = np.random.default_rng(2)
    arrays = [rng.random((5, 7, 9)).astype(np.float32) for _ in range(3)]
    sums = TripleSum((5, 7, 9), "cuda:0")(*(torch.from_numpy(a).cuda() for a in arrays))
    assert sums == pytest.approx([a.astype(np.float64).sum() for a in arrays], rel=1e-6)
