"""Replica logic of bench.py on host ranks (gloo, world size 2): the
timing reduction takes the maximum over ranks, the barrier joins, and
every rank reads its rank/world from the launcher's environment. The
path itself does not shard (independent replicas), so this is the whole
of its multi-process logic."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    import torch.distributed as dist

    r, w, local = bench.dist_setup()
    bench.barrier(w)
    # each rank's own time; the reported step time is the slowest rank's
    got = bench.max_over_ranks(10.0 + 5.0 * r, w)
    out.put((r, w, local, got))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_host_ranks_reduce_to_the_slowest():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == world for r in res)
    assert all(r[3] == pytest.approx(15.0) for r in res)
