"""Host-side sharding of independent solves across GPUs (one process per GPU).

Instances of the batched and served workloads are independent, so they are partitioned across
ranks with no collective on the data path: each rank holds a replica of the shared operators
and steps only its own instances. The only cross-rank traffic is host-side: the request
assignment (computed identically on every rank from the seeded stream) and one gather of the
per-request statistics at the end.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous balanced partition of n items: rank r gets [start, stop)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def route(costs: Sequence[float], world: int, policy: str = "least_work") -> List[int]:
    """Rank of every request, in arrival order. ``least_work`` sends each request to the rank
    with the least assigned work so far (ties to the lowest rank); ``round_robin`` cycles."""
    if world <= 0:
        raise ValueError("world must be >= 1")
    if policy == "round_robin":
        return [k % world for k in range(len(costs))]
    if policy != "least_work":
        raise ValueError(f"unknown policy {policy}")
    load = [0.0] * world
    out = []
    for c in costs:
        r = min(range(world), key=lambda j: (load[j], j))
        load[r] += float(c)
        out.append(r)
    return out


def gather(obj, group=None) -> Optional[list]:
    """All ranks' objects on every rank (torch.distributed, any backend); [obj] when not distributed."""
    try:
        import torch.distributed as dist
    except Exception:
        return [obj]
    if not dist.is_available() or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out


def serve_sharded(costs: Sequence[float], rank: int, world: int, serve_share: Callable[[List[int]], list],
                  policy: str = "least_work") -> list:
    """Runs one request stream across ranks with no data-path collective.

    ``costs`` is the stream in arrival order (identical on every rank, e.g. the request step
    counts). Each request is routed to a rank (``route``); this rank passes the global indices
    of its share to ``serve_share``, which serves them (on this rank's GPU) and returns one
    record per index, in the order given. The records of all ranks are then gathered once and
    returned on every rank in arrival order, each with its ``rank`` and ``index`` added. A rank
    that fails raises before the gather; the other ranks' gather then ends with the process
    group's timeout error instead of waiting for good.
    """
    ranks = route(costs, world, policy)
    mine = [k for k, r in enumerate(ranks) if r == rank]
    recs = serve_share(mine)
    if len(recs) != len(mine):
        raise RuntimeError(f"rank {rank}: {len(recs)} records for {len(mine)} requests")
    local = [dict(rec, rank=rank, index=k) for k, rec in zip(mine, recs)]
    allv = gather(local) or [local]
    merged = [rec for part in allv for rec in part]
    merged.sort(key=lambda r: r["index"])
    if [r["index"] for r in merged] != list(range(len(costs))):
        raise RuntimeError("gathered records do not cover the stream exactly once")
    return merged
