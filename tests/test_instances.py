"""Instance sharding for several GPUs: the assignment is a disjoint cover balanced by cost, and the gloo
gather gives every rank every instance's result (world size 2, CPU processes)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from plume_b200.sim.instances import assign_instances, instance_cost, max_over_ranks, run_instances


def test_assignment_is_a_balanced_disjoint_cover():
    costs = [5.0, 1.0, 4.0, 4.0, 2.0, 3.0, 8.0]
    shares = assign_instances(costs, 3)
    flat = sorted(i for share in shares for i in share)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in share) for share in shares]
    assert max(loads) - min(loads) <= max(costs)
    assert assign_instances(costs, 3) == shares  # deterministic
    assert assign_instances([], 2) == [[], []]
    with pytest.raises(ValueError):
        assign_instances(costs, 0)


def test_instance_cost_counts_cells_times_substeps():
    from plume_b200.recipe.derived import derive
    from plume_b200.workloads import smoke_puff_recipe

    recipe = smoke_puff_recipe((16, 24, 16), frames=5)
    assert instance_cost(recipe, derive(recipe)) == 16 * 24 * 16 * 5


def _worker(rank: int, world: int, port: int, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ran = []

        def run(index):
            ran.append(index)
            return {"instance": index, "rank": rank, "cost": costs[index]}

        results = run_instances(len(costs), costs, run)
        slowest = max_over_ranks(float(rank + 1))
        out.put((rank, sorted(ran), {k: v["rank"] for k, v in results.items()}, slowest))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_share_the_instances_and_gather_all_results():
    costs = [3.0, 9.0, 1.0, 7.0, 2.0]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, out)) for r in range(2)]
    for p in procs:
        p.start()
    reports = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {rank: (ran, owners, slowest) for rank, ran, owners, slowest in reports}
    shares = assign_instances(costs, 2)
    assert by_rank[0][0] == shares[0] and by_rank[1][0] == shares[1]
    for rank in (0, 1):
        owners = by_rank[rank][1]
        assert sorted(owners) == list(range(len(costs)))
        assert all(owners[i] == (0 if i in shares[0] else 1) for i in owners)
        assert by_rank[rank][2] == 2.0  # the max over ranks
