"""Scenario sharding across ranks (one process per GPU).

Scenarios are independent, so a batch splits into contiguous blocks with no
collective on the data path.  The only exchange is the batch sum of
parameters shared by all scenarios (1-D roughness r[L] or emitter Ke[N]):
the reference returns their gradient summed over the batch
(dgga/autodiff.py:1306-1308), which across ranks is one SUM all-reduce.
"""
from __future__ import annotations


def scenario_shard(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of this rank's contiguous block; block sizes differ by
    at most one and cover 0..n_total-1 exactly once."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world: %d/%d" % (rank, world))
    base, extra = divmod(int(n_total), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def allreduce_batch_summed(grads, group=None):
    """In-place SUM all-reduce of batch-summed parameter gradients (NCCL on
    GPUs, gloo on CPU).  A no-op outside an initialised process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return grads
    for g in grads:
        if g is not None:
            dist.all_reduce(g, op=dist.ReduceOp.SUM, group=group)
    return grads
