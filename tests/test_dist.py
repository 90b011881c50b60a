"""Replica plumbing of bench.py on two CPU ranks (gloo): the timing of the
slowest rank is what every rank reports, and barriers line the ranks up.
The engine itself is one GPU per process with no data exchange."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    ws, r, local = bench.dist_init()
    assert (ws, r) == (world, rank)
    bench.barrier(ws)
    t = bench.max_over_ranks(10.0 + rank, ws, local)
    out[rank] = t
    import torch.distributed as dist
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_max_timing():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
        assert p.exitcode == 0
    assert out[0] == out[1] == 11.0
