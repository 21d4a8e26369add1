"""Replicas on several GPUs (one process per GPU): the raw-WAH path shards as
independent operand pairs, so ranks share no data; the only exchanges are
the timing reductions.  Used by bench.py; the functions take the process
group's backend as it is (NCCL on GPUs, gloo in the CPU tests)."""
from __future__ import annotations


def operand_seeds(rank: int, ndensities: int):
    """(seed of A, seed of B) per density for this rank: every rank builds
    its own pairs, disjoint from every other rank's."""
    return [(1000 * rank + 2 * i + 1, 1000 * rank + 2 * i + 2) for i in range(ndensities)]


def max_over_ranks(ms: float, device=None) -> float:
    """The largest of every rank's device time (all ranks must call it)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(bytes_per_rank: int, steps: int, ms_max: float, world: int) -> float:
    """GB/s of the whole job: every rank moved bytes_per_rank per step, the
    slowest rank's time bounds the job."""
    return world * bytes_per_rank * steps / (ms_max / 1e3) / 1e9
