"""The mixed-precision step: velocity, smoke and temperature stored as bfloat16 or float16 with float32
arithmetic (pressure and divergence float32). Checked against the FP64 oracle (the plain method in double
precision) on the same seeded state, next to the float32 step's own error, with tolerances stated per storage
type: a few storage ulps of each field's range after several substeps."""

import numpy as np
import pytest

from oracle import oracle as O
from plume_b200.recipe.derived import derive
from plume_b200.workloads import operator_fields, plain_step_recipe
from support import FIELDS, host

pytestmark = pytest.mark.gpu

# max |gpu - fp64| / max |fp64| per field after SUBSTEPS substeps (float32 storage is ~1e-6)
SUBSTEPS = 4
FIELD_TOL = {"float32": 1e-4, "bfloat16": 3e-2, "float16": 4e-3}
# max |thickness - fp64 thickness| of a rendered frame of that state (measured on B200: float32 7.6e-4,
# bfloat16 2.4e-3, float16 9.7e-4; the field errors: float32 6e-5, bfloat16 1.5e-2, float16 1.9e-3)
THICKNESS_TOL = {"float32": 2e-3, "bfloat16": 5e-3, "float16": 2e-3}


def storage_dtype(name):
    import torch

    return getattr(torch, name)


def run_pair(storage_name, cells=(24, 32, 24), substeps=SUBSTEPS):
    import torch

    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper

    recipe = plain_step_recipe(cells, cycles=4)
    derived = derive(recipe)
    d = recipe.domain
    o = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k, "f64")
    c = make_grid(derived, d.cell_m, d.faces, d.ambient_k, "cuda:0", storage=storage_dtype(storage_name))
    for name, values in operator_fields(derived.cells, 11, d.ambient_k).items():
        getattr(o, name).data[...] = values
        getattr(c, name).data.copy_(torch.from_numpy(values))
    os_, cs = O.Stepper(o, recipe), Stepper(c, recipe)
    for n in range(substeps):
        os_.step(n * derived.dt_s, derived.dt_s)
        cs.step(n * derived.dt_s, derived.dt_s)
    return recipe, derived, o, c


def field_errors(o, c):
    errors = {}
    for name in FIELDS:
        got = host(getattr(c, name).data.float()).astype(np.float64)
        want = getattr(o, name).data
        errors[name] = float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-30))
    return errors


@pytest.mark.parametrize("storage", ["float32", "bfloat16", "float16"])
def test_mixed_step_tracks_the_fp64_oracle(cuda_device, storage):
    _, _, o, c = run_pair(storage)
    assert c.smoke.data.dtype == storage_dtype(storage)
    assert c.pressure.dtype == storage_dtype("float32")
    errors = field_errors(o, c)
    print(storage, {k: f"{v:.2e}" for k, v in errors.items()})
    for name, error in errors.items():
        assert error < FIELD_TOL[storage], f"{storage} {name}: {error:.3g}"


@pytest.mark.parametrize("storage", ["float32", "bfloat16", "float16"])
def test_mixed_frame_tracks_the_fp64_oracle(cuda_device, storage):
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer

    recipe, derived, o, c = run_pair(storage)
    view = sheet_domain_view(recipe, derived)
    frame = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "cuda:0").render(c)
    expected = O.FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, "f64").render(o)
    error = float(np.abs(frame[..., 1] - expected[..., 1]).max())
    print(storage, f"thickness {error:.2e}", f"max thickness {float(expected[..., 1].max()):.3f}")
    assert error < THICKNESS_TOL[storage]


def test_mixed_storage_is_deterministic(cuda_device):
    import torch

    first = run_pair("bfloat16", substeps=2)[3]
    second = run_pair("bfloat16", substeps=2)[3]
    for name in FIELDS:
        assert torch.equal(getattr(first, name).data, getattr(second, name).data), name
