"""Field-level partition of the batched and served forms across GPUs.

Fields are independent: a correction reads and writes only its own two
fields, so a multi-GPU batch needs no collective on the data path.  A host
scheduler assigns each field to one rank (one process per GPU), every rank
corrects its share with ``extremz_correct_batch`` on its own device, and only
the reports travel, gathered on the host (``all_gather_object`` of the
process group).  The corrected fields stay where they were corrected.

The reference corrects one field per process run (``main.cpp:65-446``); this
module is the multi-GPU form of the batched call above it.  One field is not
split (its steepest-path labels are global; the reference's unfinished
z-slab scheme is ``src/distributed_ExtreM.cu:256-608``).

Scheduling
----------
A correction's device time grows with the field's voxel count (the setup and
every dense pass are linear in it; the rounds are incremental), so the static
plan balances voxels: longest-processing-time first -- fields in descending
size (ties by index) each to the rank with the least load so far (ties to the
lower rank).  Its makespan is within 4/3 of the optimum.  Requests of the
served form arrive one at a time; ``route`` sends each to the rank with the
fewest outstanding voxels.
"""

from __future__ import annotations

import heapq
from typing import List, Sequence


def plan(voxels: Sequence[int], n_ranks: int) -> List[List[int]]:
    """Partition field indices over ``n_ranks`` ranks by voxel count
    (longest first to the least-loaded rank).  Every index appears once; each
    rank's list is in ascending index order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    order = sorted(range(len(voxels)), key=lambda i: (-int(voxels[i]), i))
    heap = [(0, r) for r in range(n_ranks)]
    parts: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(voxels[i]), r))
    return [sorted(p) for p in parts]


def loads(voxels: Sequence[int], parts: Sequence[Sequence[int]]) -> List[int]:
    """Voxels per rank under a plan."""
    return [sum(int(voxels[i]) for i in p) for p in parts]


def route(outstanding: Sequence[int]) -> int:
    """The rank a new request goes to: the fewest outstanding voxels, ties to
    the lower rank."""
    if not outstanding:
        raise ValueError("no ranks")
    return min(range(len(outstanding)), key=lambda r: (outstanding[r], r))


def correct_batch_sharded(ctx, items, voxels: Sequence[int], *, rank: int, world: int,
                          group=None, stream=None):
    """Correct this rank's share of a batch and gather every field's report.

    items: the whole batch as ``Context.correct_batch`` takes it; a rank only
    touches the entries the plan gives it (the others may be None), so each
    rank needs device tensors for its own fields only.  voxels: each field's
    voxel count (the same on every rank, so every rank computes the same
    plan).  Returns (reports of all fields in batch order, the plan, this
    rank's kernel launches).  With world == 1 no process group is needed.
    """
    parts = plan(voxels, world)
    mine = parts[rank]
    reps, launches = ctx.correct_batch([items[i] for i in mine], stream=stream) if mine else ([], 0)
    shares = [(mine, reps)]
    if world > 1:
        import torch.distributed as dist
        shares = [None] * world
        dist.all_gather_object(shares, (mine, reps), group=group)
    out = [None] * len(voxels)
    for idx, rs in shares:
        for i, r in zip(idx, rs):
            out[i] = r
    if any(r is None for r in out):
        raise RuntimeError("a field of the batch has no report")
    return out, parts, launches


class Router:
    """Requests over several devices' servers, each to the one with the fewest
    outstanding voxels (``route``).

    servers: one ``api.Server`` per device (or any object with the same
    ``submit(f, decp, bound, **kw) -> ticket`` / ``poll(ticket)`` /
    ``wait(ticket, timeout_ms)`` calls).  A request's tensors must live on
    the device of the server it goes to, so the caller asks ``pick`` first and
    places the request there; ``submit`` then queues it.  Tickets are the
    router's own, (server index, server ticket) inside.
    """

    def __init__(self, servers):
        if not servers:
            raise ValueError("no servers")
        self.servers = list(servers)
        self.outstanding = [0] * len(self.servers)
        self._open = {}  # router ticket -> (server, server ticket, voxels)
        self._next = 0

    def pick(self, voxels: int) -> int:
        """The server index the next request of ``voxels`` voxels goes to."""
        return route(self.outstanding)

    def submit(self, index: int, f, decp, bound: float, **kw) -> int:
        voxels = int(f.numel())
        t = self.servers[index].submit(f, decp, bound, **kw)
        self.outstanding[index] += voxels
        tk = self._next
        self._next += 1
        self._open[tk] = (index, t, voxels)
        return tk

    def _done(self, tk, res):
        if res is not None:
            index, _, voxels = self._open.pop(tk)
            self.outstanding[index] -= voxels
        return res

    def poll(self, tk: int):
        """None while pending, else the server's (report, latency ms)."""
        index, t, _ = self._open[tk]
        return self._done(tk, self.servers[index].poll(t))

    def wait(self, tk: int, timeout_ms: int = -1):
        index, t, _ = self._open[tk]
        return self._done(tk, self.servers[index].wait(t, timeout_ms))
