"""The batched frame loop (many recipes on one GPU, one stream each) gives every instance exactly the bytes
and step counts of running it alone through simulate_frames."""

import pytest

from plume_b200.workloads import batched_recipes, operator_fields

pytestmark = pytest.mark.gpu

SMALL_GRIDS = ((16, 16, 16), (24, 32, 24), (20, 28, 16))


def seeded(index, grid):
    """Seeded fields, velocities scaled up so that the CFL cap splits some frames into more substeps."""
    import torch

    fields = operator_fields(grid.cells, 100 + index, 1.0)
    for name, values in fields.items():
        scale = 12.0 if name in ("u", "v", "w") else 1.0
        getattr(grid, name).data.copy_(torch.from_numpy(values * scale).to(grid.storage))


@pytest.mark.parametrize("storage", ["float32", "bfloat16"])
def test_batch_matches_one_at_a_time(cuda_device, storage):
    import torch

    from plume_b200.sim.batch import Batch, run_one_at_a_time

    dtype = getattr(torch, storage)
    recipes = batched_recipes(count=6, frames=4, seed=5, grids=SMALL_GRIDS)
    alone = {}

    def keep(index, frame, grid):
        alone[(index, frame)] = {name: getattr(grid, name).data.clone() for name in ("u", "smoke", "temperature")}

    logs_alone = run_one_at_a_time(recipes, "cuda:0", storage=dtype, initial_state=seeded, capture=keep)
    together = {}

    def keep_batched(index, frame, grid):
        together[(index, frame)] = {name: getattr(grid, name).data.clone() for name in ("u", "smoke", "temperature")}

    batch = Batch(recipes, "cuda:0", storage=dtype, initial_state=seeded)
    logs_batched = batch.run(capture=keep_batched)
    torch.cuda.synchronize()
    assert logs_batched == logs_alone
    assert sorted(together) == sorted(alone)
    for key, fields in alone.items():
        for name, values in fields.items():
            assert torch.equal(together[key][name], values), (key, name)
    assert any(log.added_steps > 0 for log in logs_alone)  # the CFL cap split some blocks


def test_batch_waits_for_its_setup_on_a_delayed_stream(cuda_device):
    """The instances' streams start only after the grid, the stepper's levels and scratch and the speed slot
    are filled on the current stream: with that stream held busy while the batch is built, the batch still
    gives the bytes and step counts of running each recipe alone."""
    import torch

    from plume_b200.sim.batch import Batch, run_one_at_a_time

    recipes = batched_recipes(count=3, frames=3, seed=9, grids=SMALL_GRIDS)
    alone, together = {}, {}
    logs_alone = run_one_at_a_time(recipes, "cuda:0", initial_state=seeded,
                                   capture=lambda i, f, g: alone.__setitem__((i, f), g.smoke.data.clone()))
    torch.cuda.synchronize()
    torch.cuda._sleep(200_000_000)  # keeps the current stream busy for tens of milliseconds
    batch = Batch(recipes, "cuda:0", initial_state=seeded)
    logs = batch.run(capture=lambda i, f, g: together.__setitem__((i, f), g.smoke.data.clone()))
    torch.cuda.synchronize()
    assert logs == logs_alone
    for key, values in alone.items():
        assert torch.equal(together[key], values), key


def test_a_reset_batch_repeats_its_run_in_either_schedule(cuda_device):
    """Batch.reset puts every instance back at its start: a second run, concurrent or one instance after
    another, gives the first run's step counts and frames byte for byte."""
    import torch

    from plume_b200.sim.batch import Batch

    recipes = batched_recipes(count=4, frames=3, seed=11, grids=SMALL_GRIDS)
    runs = []
    batch = Batch(recipes, "cuda:0", initial_state=seeded)
    for sequential in (False, True, False):
        frames = {}
        logs = batch.run(capture=lambda i, f, g: frames.__setitem__((i, f), g.smoke.data.clone()),
                         sequential=sequential)
        torch.cuda.synchronize()
        runs.append((logs, frames))
        batch.reset()
    for logs, frames in runs[1:]:
        assert logs == runs[0][0]
        assert sorted(frames) == sorted(runs[0][1])
        for key, values in runs[0][1].items():
            assert torch.equal(frames[key], values), key
