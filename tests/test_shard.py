"""Field-level partition of the batched form across ranks (extrem_z_b200.shard).

The plan must give every field to exactly one rank, the same plan on every
rank, and a makespan within the longest-processing-time bound; the sharded
batch must gather every field's report in batch order; the request router
must send each request to the server with the fewest outstanding voxels and
release them on completion.  The multi-rank gather runs on two CPU ranks
(gloo) with a stand-in for the correction context that records which fields
it was handed; the router runs over stand-in servers.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from extrem_z_b200 import shard, synth


def test_plan_gives_every_field_to_one_rank():
    rng = np.random.default_rng(3)
    vox = [int(v) for v in rng.integers(1, 10 ** 6, size=64)]
    for n in (1, 2, 3, 4, 8):
        parts = shard.plan(vox, n)
        assert len(parts) == n
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(vox)))
        assert all(p == sorted(p) for p in parts)
        assert shard.plan(vox, n) == parts  # deterministic


def test_plan_makespan_within_lpt_bound():
    rng = np.random.default_rng(4)
    for n in (2, 4, 8):
        vox = [int(v) for v in rng.integers(1, 10 ** 6, size=200)]
        ld = shard.loads(vox, shard.plan(vox, n))
        lower = max(sum(vox) / n, max(vox))  # no schedule beats this
        assert max(ld) <= 4.0 / 3.0 * lower + 1
        assert sum(ld) == sum(vox)


def test_plan_mixed_batch_balances_voxels():
    specs = synth.mixed_batch_specs(64)
    vox = [s["w"] * s["h"] * s["d"] for s in specs]
    ld = shard.loads(vox, shard.plan(vox, 4))
    assert max(ld) - min(ld) <= max(vox)


def test_plan_more_ranks_than_fields():
    parts = shard.plan([5, 3], 4)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1]
    with pytest.raises(ValueError):
        shard.plan([1], 0)


def test_route_takes_the_least_loaded_rank():
    assert shard.route([5, 2, 2, 9]) == 1
    assert shard.route([0]) == 0
    with pytest.raises(ValueError):
        shard.route([])


class _FakeCtx:
    """Stands in for api.Context: 'corrects' by reporting the field's tag."""

    def __init__(self, rank):
        self.rank = rank

    def correct_batch(self, items, stream=None):
        return [{"tag": it[0], "rank": self.rank} for it in items], 7 * len(items)


def test_single_rank_needs_no_process_group():
    items = [(i, None, 0.1) for i in range(5)]
    reps, parts, launches = shard.correct_batch_sharded(_FakeCtx(0), items, [3, 1, 4, 1, 5],
                                                        rank=0, world=1)
    assert [r["tag"] for r in reps] == list(range(5))
    assert parts == [[0, 1, 2, 3, 4]] and launches == 35


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, vox, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    # Each rank holds only its own fields: the others are None.
    parts = shard.plan(vox, world)
    items = [(i, None, 0.1) if i in parts[rank] else None for i in range(len(vox))]
    reps, got, launches = shard.correct_batch_sharded(_FakeCtx(rank), items, vox, rank=rank,
                                                      world=world)
    out[rank] = ([r["tag"] for r in reps], [r["rank"] for r in reps], got, launches)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_sharded_batch_gathers_reports_in_batch_order_on_gloo():
    world = 2
    vox = [64 ** 3, 32 ** 3, 48 ** 3, 16 ** 3, 40 ** 3, 24 ** 3, 56 ** 3]
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, vox, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    parts = shard.plan(vox, world)
    owner = {i: r for r, p in enumerate(parts) for i in p}
    for rank in range(world):
        tags, ranks, got, launches = out[rank]
        assert tags == list(range(len(vox)))
        assert ranks == [owner[i] for i in range(len(vox))]
        assert got == parts
        assert launches == 7 * len(parts[rank])


class _FakeTensor:
    def __init__(self, n):
        self.n = n

    def numel(self):
        return self.n


class _FakeServer:
    """Completes a request when told to; reports the voxels it saw."""

    def __init__(self):
        self.jobs, self.done = {}, set()

    def submit(self, f, decp, bound, **kw):
        t = len(self.jobs)
        self.jobs[t] = f.numel()
        return t

    def poll(self, t):
        return ({"voxels": self.jobs[t]}, 1.0) if t in self.done else None

    def wait(self, t, timeout_ms=-1):
        self.done.add(t)
        return self.poll(t)


def test_router_balances_outstanding_voxels_and_releases_them():
    srv = [_FakeServer(), _FakeServer(), _FakeServer()]
    router = shard.Router(srv)
    tickets = []
    for n in (900, 500, 400, 300, 300):
        i = router.pick(n)
        tickets.append((router.submit(i, _FakeTensor(n), None, 0.1), i, n))
    # 900 -> 0, 500 -> 1, 400 -> 2, 300 -> 2 (400 < 500), 300 -> 1 (500 < 700).
    assert [i for _, i, _ in tickets] == [0, 1, 2, 2, 1]
    assert router.outstanding == [900, 800, 700]
    tk, i, n = tickets[0]
    assert router.poll(tk) is None
    rep, ms = router.wait(tk)
    assert rep["voxels"] == 900 and router.outstanding == [0, 800, 700]
    assert router.pick(100) == 0
    with pytest.raises(ValueError):
        shard.Router([])
