"""The multi-rank plumbing of bench.py (one process per GPU; barrier and the
max-over-ranks of the timed region) on two CPU ranks over gloo."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import sys

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    d = bench.Dist(world)
    d.barrier()
    t = d.max(0.5 + rank)  # rank 1 is the slow one
    links, steps = 4 * 32 ** 4, 10
    value = d.world * links * steps / t
    d.close()
    q.put((rank, t, value))


def test_two_ranks_take_the_max_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [1.5, 1.5]           # every rank sees the slowest rank's time
    assert res[0][2] == pytest.approx(2 * 4 * 32 ** 4 * 10 / 1.5)  # whole-job link-updates/s
