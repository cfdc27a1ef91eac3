"""View sharding across ranks (one process per GPU).

Rays are independent, so a multiview acquisition shards by view: every rank keeps a
resident copy of the field, projects and differentiates its own contiguous block of
views, and the only exchange is the sum of the per-rank volume gradients (one
all-reduce; NCCL over NVLink on GPUs, gloo in the CPU tests).  Pose gradients are per
view and stay on their rank.
"""

from __future__ import annotations

from .contracts import ContractError


def view_range(views: int, rank: int, world: int) -> range:
    """Contiguous block of views owned by ``rank`` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world or views < world:
        raise ContractError("need at least one view per rank and 0 <= rank < world")
    base, extra = divmod(views, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def reduce_volume_gradient(gradient, group=None):
    """Sum a rank's volume gradient over all ranks, in place (no-op without a process group)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(gradient, op=dist.ReduceOp.SUM, group=group)
    return gradient
