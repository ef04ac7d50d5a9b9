"""Ensembles across GPUs: one process per GPU, members partitioned across the
ranks, no collective while stepping, one gather of per-member results at the
end.

The members of an ensemble are independent, so the only exchange is the final
gather (host side, through torch.distributed's object collectives: gloo or
NCCL).  The partition balances the work, estimated as cells x steps, by the
longest-processing-time rule: members in decreasing cost order, each to the
least loaded rank (ties to the lowest rank), so every rank computes the same
partition without communicating.
"""
from typing import Callable, List, Sequence


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Member indices per rank (each list in increasing index order)."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def member_cost(params, steps: int) -> float:
    r = params.rec
    return float(r.Nx * r.Ny * r.Nz) * steps


def run_sharded(n_members: int, costs: Sequence[float], run_members: Callable[[List[int]], list], group=None):
    """Run this rank's share and gather every member's result on rank 0.

    run_members(indices) steps the given members on this rank's GPU and
    returns one picklable result per index, in the same order.  Returns the
    results of all members in member order on rank 0 and None elsewhere (or
    the local results when torch.distributed is not initialised)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return run_members(list(range(n_members)))
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = partition(costs, world)[rank]
    local = run_members(mine)
    if len(local) != len(mine):
        raise RuntimeError("run_members returned %d results for %d members" % (len(local), len(mine)))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, local)), gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * n_members
    for part in gathered:
        for i, res in part:
            out[i] = res
    return out


def ensemble_runner(built, steps: int, precision: str = "fp32"):
    """run_members for run_sharded: builds this rank's members on the current
    CUDA device, steps them together and returns their FP64 diagnostics."""
    def run(indices):
        from . import Ensemble
        if not indices:
            return []
        with Ensemble([built[i][0] for i in indices], precision) as ens:
            for q, i in enumerate(indices):
                ens[q].upload(built[i][1], built[i][2])
            ens.step(steps)
            ens.synchronize()
            return [ens[q].diagnostics(allow_nan=True) for q in range(len(indices))]
    return run
