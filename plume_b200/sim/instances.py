"""Independent simulation instances over several GPUs (one process per GPU).

A single grid does not shard: every stencil pass and every multigrid level would need a halo exchange. Many
recipes (preview variants, parameter sweeps) are independent, so they are assigned whole to ranks -- greedy
longest-first by estimated cost (cells x substeps) -- and each rank runs its share with no exchange on the
data path; only the per-instance results travel, once, over torch.distributed (gloo or NCCL).
"""

from collections.abc import Callable, Sequence

import torch.distributed as dist


def instance_cost(recipe, derived) -> float:
    """Estimated work of one instance: cells x base substeps (warmup included)."""
    nx, ny, nz = derived.cells
    return float(nx * ny * nz) * (derived.warmup_steps + derived.steps_per_frame * recipe.time.frames)


def assign_instances(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Instance indices per rank: longest first, each to the currently lightest rank (ties: lowest rank)."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    loads = [0.0] * world_size
    shares: list[list[int]] = [[] for _ in range(world_size)]
    for index in sorted(range(len(costs)), key=lambda n: (-costs[n], n)):
        rank = min(range(world_size), key=lambda r: (loads[r], r))
        shares[rank].append(index)
        loads[rank] += costs[index]
    return [sorted(share) for share in shares]


def run_instances(count: int, costs: Sequence[float], run: Callable[[int], object]) -> dict[int, object]:
    """Runs this rank's share of `count` instances (`run(index)` returns the instance's result) and returns
    every instance's result on every rank. Without an initialised process group everything runs here."""
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    mine = {index: run(index) for index in assign_instances(costs, world)[rank]}
    if world == 1:
        return mine
    gathered: list[dict] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(gathered, mine)
    results: dict[int, object] = {}
    for part in gathered:
        results.update(part)
    if sorted(results) != list(range(count)):
        raise RuntimeError("instance results are missing after the gather")
    return results


def max_over_ranks(value: float) -> float:
    """The largest value over all ranks (the timing rule for multi-GPU numbers)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    import torch

    backend = dist.get_backend()
    device = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
