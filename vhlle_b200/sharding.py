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


# --------------------------------------------------------------- one event, many GPUs
# A single event split along eta into one slab per rank.  A step reaches at
# most HALO cells along eta, so a slab that stores HALO extra planes beyond
# each inner edge, refreshed from its neighbours' owned planes once per
# step, evolves its owned planes bit for bit as the whole grid does (its own
# ghost-cell copies at an inner edge touch only halo planes that the next
# exchange overwrites).  The exchange is one send and one receive per inner
# edge of HALO planes x every persistent field (vh_pack_planes /
# vh_unpack_planes on the device; NCCL send/recv between the GPUs).
HALO = 6


def slab_ranges(nz: int, world: int, halo: int = HALO) -> List[Tuple[int, int, int, int]]:
    """Per rank (owned z0, owned z1, stored z0, stored z1): owned planes
    split as evenly as possible, each slab stored with `halo` more planes on
    every side that has a neighbour."""
    if world < 1 or nz < world * max(halo, 1):
        raise ValueError("cannot split %d eta cells among %d ranks with %d halo planes "
                         "(every slab must own at least as many planes as a halo)"
                         % (nz, world, halo))
    bounds = [nz * r // world for r in range(world + 1)]
    out = []
    for r in range(world):
        a, b = bounds[r], bounds[r + 1]
        out.append((a, b, max(0, a - halo), min(nz, b + halo)))
    return out


def slab_grid(grid, z0: int, z1: int):
    """The Grid of planes [z0, z1) of `grid`: its eta bounds are the planes'
    coordinates (Fluid::getZ of the whole grid) and its cell size is the
    whole grid's, bit for bit."""
    from . import workloads as W
    dz = grid.dz
    return W.Grid(grid.nx, grid.ny, z1 - z0, grid.xmin, grid.xmax, grid.ymin, grid.ymax,
                  grid.etamin + z0 * dz, grid.etamin + (z1 - 1) * dz, cell_dz=dz)


def slab_setup(setup, z0: int, z1: int):
    """The Setup of planes [z0, z1) of an event (initial Q and m sliced)."""
    import copy
    g = setup.grid
    nxy = g.nx * g.ny
    s = copy.copy(setup)
    s.grid = slab_grid(g, z0, z1)
    s.Q = setup.Q.reshape(7, g.nz, nxy)[:, z0:z1].reshape(7, -1).copy()
    s.m = setup.m.reshape(g.nz, nxy)[z0:z1].reshape(-1).copy()
    if setup.pi is not None:
        s.pi = setup.pi.reshape(10, g.nz, nxy)[:, z0:z1].reshape(10, -1).copy()
    if setup.Pi is not None:
        s.Pi = setup.Pi.reshape(g.nz, nxy)[z0:z1].reshape(-1).copy()
    s.name = "%s_slab_%d_%d" % (setup.name, z0, z1)
    return s


def halo_plan(ranges, rank: int):
    """The exchanges of `rank`, lower neighbour first: (peer, send z0 and
    planes (local), receive z0 and planes (local)).  What a rank sends is
    the part of its owned planes its neighbour stores as halo; what it
    receives fills its own halo."""
    a, b, c, d = ranges[rank]
    plan = []
    if rank > 0:
        dp = ranges[rank - 1][3]
        plan.append((rank - 1, a - c, dp - a, 0, a - c))
    if rank < len(ranges) - 1:
        an, _, cn, _ = ranges[rank + 1]
        plan.append((rank + 1, cn - c, an - cn, b - c, d - b))
    return plan


def exchange_halos(dist, ranges, rank: int, pack, unpack, new_buffer) -> None:
    """One halo exchange of `rank` with its neighbours through torch
    distributed point-to-point calls (NCCL between GPUs, gloo on the host):
    pack(z0, n, buf) / unpack(z0, n, buf) move planes between the slab and a
    buffer from new_buffer(n).  Every send and receive is posted before any
    is waited on, so the ranks cannot deadlock."""
    ops, recvs = [], []
    for peer, z_send, n_send, z_recv, n_recv in halo_plan(ranges, rank):
        sbuf, rbuf = new_buffer(n_send), new_buffer(n_recv)
        pack(z_send, n_send, sbuf)
        ops.append(dist.P2POp(dist.isend, sbuf, peer))
        ops.append(dist.P2POp(dist.irecv, rbuf, peer))
        recvs.append((z_recv, n_recv, rbuf))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for z, n, buf in recvs:
        unpack(z, n, buf)


def slab_window(ranges, rank: int, nz: int):
    """vh_set_slab's arguments for `rank`'s slab of a grid of nz planes:
    (owned z0, owned z1 in its own planes, its first plane in the grid, nz)."""
    a, b, c, _ = ranges[rank]
    return a - c, b - c, c, nz


def merge_slab_surfaces(parts):
    """The whole grid's freeze-out records from its slabs' (records [n][29],
    cells [n][3]) pairs, in slab order: Fluid::outputSurface visits the
    hypercubes ix-, iy-, then iz-ordered (iz fastest) and writes each cube's
    elements in turn, so a stable sort of the concatenated records by their
    cube's (ix, iy, iz) restores its order."""
    import numpy as np
    if not parts:
        return np.zeros((0, 29))
    rec = np.concatenate([p[0] for p in parts])
    cells = np.concatenate([np.asarray(p[1]).reshape(-1, 3) for p in parts])
    order = np.lexsort((cells[:, 2], cells[:, 1], cells[:, 0]))  # stable
    return rec[order]


def merge_slab_totals(parts):
    """The whole grid's totals from its slabs' (vh_totals dicts): every
    entry is a sum over the owned interior cells."""
    out = {}
    for t in parts:
        for k, v in t.items():
            out[k] = out.get(k, 0.0) + v
    return out
