"""bench.py's N > 1 host logic on CPU: two gloo ranks take disjoint batch ids
of one experiment and agree on the slowest rank's time (the multi-GPU run
is replicas with no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, steps, out):
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batches = [bench.batch_of(s, rank, world) for s in range(steps)]
        slowest = bench.max_over_ranks(10.0 + rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, batches)
        out.put((rank, batches, slowest, gathered))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replicas_take_disjoint_batches(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    steps = 5
    procs = [ctx.Process(target=rank_main, args=(r, world, port, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, batches, slowest, gathered in results:
        assert slowest == 10.0 + world - 1               # every rank sees the max
        flat = [b for g in gathered for b in g]
        assert len(flat) == len(set(flat)) == world * steps   # disjoint, none skipped
        assert sorted(flat) == list(range(world * steps))


def test_single_rank_needs_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert [bench.batch_of(s, 0, 1) for s in range(4)] == [0, 1, 2, 3]
