"""Event sharding across GPUs: one process per GPU, each evolving its own
events; there is no exchange on the data path (events are independent), so
the only collectives are host-side: a barrier around the timed region, the
max of the per-rank device times, and a gather of the per-event results
(totals, surface counts) to rank 0.  They run over torch.distributed's gloo
backend on the host, which also makes them testable without GPUs.
"""
from __future__ import annotations

import datetime
import os
from typing import Any, List, Sequence, Tuple


def dist_env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_events(cells: Sequence[int], world: int, rank: int) -> List[int]:
    """Indices of the events rank `rank` evolves: longest-processing-time
    assignment by cell count (largest event first to the least loaded rank,
    ties to the lower rank), returned in the events' original order.  Every
    event goes to exactly one rank and the result depends only on the cell
    counts, so all ranks agree without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank: %r/%r" % (world, rank))
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    owner = [0] * len(cells)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += int(cells[i])
    return [i for i in range(len(cells)) if owner[i] == rank]


class Ranks:
    """Host collectives for a sharded run (no-ops for a single process)."""

    def __init__(self, world: int | None = None, timeout_s: float = 600.0):
        self.world = dist_env()[0] if world is None else world
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def rank(self) -> int:
        return self.dist.get_rank() if self.dist else 0

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj: Any) -> List[Any] | None:
        """Every rank's object, in rank order, on rank 0 (None elsewhere)."""
        if not self.dist:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object(obj, out, dst=0)
        return out

    def close(self) -> None:
        if self.dist and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None
