"""Multi-rank plumbing of bench.py on CPU ranks (gloo, world size 2).

The correction path does not shard: with N GPUs the benchmark runs N replicas
and reports all ranks' voxels over the max-over-ranks time.  These tests run
the barrier and the max reduction bench.py uses on two CPU ranks.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      EXTREMZ_DIST_BACKEND="gloo")
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    w, r, _ = bench.dist_setup()
    assert (w, r) == (world, rank)
    bench.barrier(w)
    out[rank] = bench.max_over_ranks(10.0 * (rank + 1), w)
    import torch.distributed as dist
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_barrier_on_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    assert dict(out) == {0: 20.0, 1: 20.0}
