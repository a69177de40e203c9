"""Host logic of multi-GPU runs: independent work split across ranks.

The solver path does not shard without a halo exchange, so several GPUs run
independent work -- ensemble members, or replicas of one problem -- with no
collective on the data path.  The only communication is the reduction of the
reported numbers: the sum of the work units over ranks and the maximum of the
device times (the slowest rank sets the job's time).  One process per GPU,
launched by torchrun; the same functions run over NCCL on GPUs and over gloo
on CPU (the tests).
"""

from __future__ import annotations

from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def partition(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of ``items`` for ``rank`` (disjoint, covering, sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return list(items[rank::world])


def reduce_totals(work: float, ms: float, device=None) -> Tuple[float, float]:
    """(sum of ``work`` over ranks, max of ``ms`` over ranks); identity without an initialised process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(work), float(ms)
    w = torch.tensor([float(work)], dtype=torch.float64, device=device)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(w.item()), float(t.item())
