"""Helpers shared by the tests: grids without a recipe (as the reference's tests/support/grids.py builds them),
and the same starting state loaded into the CUDA grid and the oracle grid."""

import numpy as np

from oracle import oracle as O
from plume_b200.recipe.derived import Derived
from plume_b200.recipe.schema import FaceSettings

ALL_CLOSED = FaceSettings(bottom="closed", top="closed", left="closed", right="closed", back="closed",
                          front="closed")
OPEN = FaceSettings()  # floor closed, the rest open


def small_derived(cells=(16, 16, 16), cell_m=0.1) -> Derived:
    size = tuple(n * cell_m for n in cells)
    return Derived(cells=tuple(cells), size_m=size, domain_min_m=(-size[0] / 2, 0.0, -size[2] / 2), fps=20.0,
                   dt_s=1 / 60, warmup_steps=0, steps_per_frame=3)


def oracle_grid(cells=(16, 16, 16), cell_m=0.1, faces=ALL_CLOSED, ambient_k=293.0, precision="f32"):
    return O.make_grid(small_derived(cells, cell_m), cell_m, faces, ambient_k, precision)


def cuda_grid(cells=(16, 16, 16), cell_m=0.1, faces=ALL_CLOSED, ambient_k=293.0):
    from plume_b200.sim.grid import make_grid

    return make_grid(small_derived(cells, cell_m), cell_m, faces, ambient_k, "cuda:0")


def blob(shape, center, radius) -> np.ndarray:
    idx = np.indices(shape).astype(np.float64) + 0.5
    dist2 = sum((idx[a] - center[a]) ** 2 for a in range(3))
    return np.exp(-dist2 / (2 * radius**2))


FIELDS = ("u", "v", "w", "smoke", "temperature")


def load_state(oracle, cuda, fields: dict) -> None:
    """Copies numpy arrays (by field name; 'pressure' too) into both grids' current data."""
    import torch

    for name, values in fields.items():
        if name == "pressure":
            oracle.pressure[...] = values
            cuda.pressure.copy_(torch.from_numpy(np.ascontiguousarray(values, dtype=np.float32)))
            continue
        getattr(oracle, name).data[...] = values
        getattr(cuda, name).data.copy_(torch.from_numpy(np.ascontiguousarray(values, dtype=np.float32)))


def host(tensor) -> np.ndarray:
    return tensor.detach().cpu().numpy()


def assert_same(actual, expected, what="") -> None:
    """Equal values (IEEE equality, so -0 == +0), with a helpful report."""
    actual = np.asarray(actual)
    expected = np.asarray(expected)
    assert actual.shape == expected.shape, f"{what}: shape {actual.shape} != {expected.shape}"
    bad = ~(actual == expected)
    if bad.any():
        diff = np.abs(actual.astype(np.float64) - expected.astype(np.float64))
        where = np.unravel_index(int(np.argmax(np.where(bad, diff, -1))), actual.shape)
        raise AssertionError(f"{what}: {int(bad.sum())} of {bad.size} differ; worst at {where}: "
                             f"{actual[where]!r} vs {expected[where]!r}")


def max_rel(actual, expected, floor: float = 0.0) -> float:
    """max |a - e| / max(|e|, floor) over all elements (floor guards near-zero values)."""
    a = np.asarray(actual, dtype=np.float64)
    e = np.asarray(expected, dtype=np.float64)
    scale = np.maximum(np.abs(e), floor)
    scale = np.where(scale == 0.0, 1.0, scale)
    return float(np.max(np.abs(a - e) / scale)) if a.size else 0.0


# The end-to-end test recipe (a 1.2 m box of 0.05 m cells, one smoke puff, 4 frames in 1 s), as a table so a
# test states only what it changes; a section given as a dict is merged into that section.
TINY_TABLE = {
    "seed": 1,
    "domain": {"size_m": [1.2, 1.2, 1.2], "cell_m": 0.05},
    "time": {"duration_s": 1.0, "frames": 4},
    "emitter": [{"name": "puff", "center_m": [0.0, 0.3, 0.0], "radius_m": 0.2, "end_s": 0.5,
                 "smoke_per_s": 5.0}],
}


def tiny_recipe(**changes):
    import copy

    from plume_b200.recipe.load import fill_dependent_defaults, parse_recipe

    table = copy.deepcopy(TINY_TABLE)
    for key, value in changes.items():
        if isinstance(value, dict) and isinstance(table.get(key), dict):
            table[key].update(value)
        else:
            table[key] = value
    return fill_dependent_defaults(parse_recipe(table), "tiny")


def put(tensor, values) -> None:
    """Copies a numpy array into a CUDA tensor of the same shape (as float32, or the tensor's storage)."""
    import torch

    tensor.copy_(torch.from_numpy(np.ascontiguousarray(values, dtype=np.float32)))
