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


def _slab_rank_main(rank, world, port, q):
    import sys

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from latticeyangmills_b200 import slab_partition

    d = bench.Dist(world)
    # the id distribution of the decomposed mode: rank 0's 128 bytes reach every rank
    box = [bytes(range(128)) if rank == 0 else None]
    d.dist.broadcast_object_list(box, src=0)
    part = slab_partition(32, world, rank)
    parts = [None] * world
    d.dist.all_gather_object(parts, part)
    d.close()
    q.put((rank, box[0], parts))


def test_decomposed_mode_host_logic_on_three_ranks():
    """Three gloo ranks agree on the NCCL id bytes and on slabs that tile the
    32 time slices with consistent neighbours."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank_main, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(3))
    assert all(r[1] == bytes(range(128)) for r in res)
    parts = res[0][2]
    assert all(r[2] == parts for r in res)
    assert [p[0] for p in parts] == [0, 11, 22] and [p[1] for p in parts] == [11, 11, 10]
    assert [(p[2], p[3]) for p in parts] == [(2, 1), (0, 2), (1, 0)]
