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


# --- the halo data path on CPU ranks ------------------------------------------------
# Each gloo rank holds one time slab of a configuration (its slices plus one
# halo slice on each side), flows it with the CPU oracle one RK3 stage at a
# time, and after every stage exchanges halo slices with its neighbours on the
# library's schedule (slab_halo_plan).  Gathered, the interiors must equal the
# whole-lattice oracle flow link for link: the exchange carries exactly the
# faces the stages need.
FLOW_N = (4, 3, 2, 7)  # x, y, z, t: 7 time slices over 2 or 3 ranks, uneven slabs
FLOW_STEPS, FLOW_EPS = 3, 0.02


def _flow_rank_main(rank, world, port, q):
    import sys

    import numpy as np

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist

    from latticeyangmills_b200 import slab_halo_plan, slab_partition
    from oracle import ymoracle as yo

    dist.init_process_group("gloo")
    n = FLOW_N
    t0, nt, lower, upper = slab_partition(n[3], world, rank)
    whole = yo.gen_expiah(n, 0.4, 11)  # (t, z, y, x, 4, 18)
    local = np.ascontiguousarray(np.concatenate([whole[(t0 - 1) % n[3]][None], whole[t0:t0 + nt],
                                                 whole[(t0 + nt) % n[3]][None]]))
    ln = (n[0], n[1], n[2], nt + 2)
    Z = np.zeros_like(local)
    peer = {"lower": lower, "upper": upper}
    for _ in range(FLOW_STEPS):
        for stage in range(3):
            yo.flow_stage(local, Z, ln, FLOW_EPS, stage)  # interior slices exact, halos stale
            reqs, bufs = [], []
            for tr in slab_halo_plan(nt):
                reqs.append(dist.isend(torch.from_numpy(local[tr["send_slice"]].copy()), peer[tr["to"]],
                                       tag=tr["tag"]))
                buf = torch.empty(local[0].shape, dtype=torch.float64)
                # the neighbour's send of the same plan entry lands here
                reqs.append(dist.irecv(buf, peer[tr["from"]], tag=tr["tag"]))
                bufs.append((tr["recv_slice"], buf))
            for r in reqs:
                r.wait()
            for sl, buf in bufs:
                local[sl] = buf.numpy()
    parts = [None] * world
    dist.all_gather_object(parts, (t0, local[1:nt + 1].copy()))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        got = np.concatenate([p[1] for p in sorted(parts, key=lambda p: p[0])])
        want = whole.copy()
        for _ in range(FLOW_STEPS):
            yo.flow(want, n, FLOW_EPS, 1, 0)
        q.put(float(np.abs(got - want).max()))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_halo_exchange_reproduces_the_whole_lattice_flow(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_flow_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    assert q.get(timeout=10) == 0.0  # bit for bit


def test_halo_plan_pairs_every_send_with_a_receive():
    from latticeyangmills_b200 import slab_halo_plan

    for nt in (1, 2, 5):
        plan = slab_halo_plan(nt)
        assert [(tr["send_slice"], tr["to"]) for tr in plan] == [(1, "lower"), (nt, "upper")]
        assert [(tr["recv_slice"], tr["from"]) for tr in plan] == [(nt + 1, "upper"), (0, "lower")]
        # what a rank sends down arrives in its lower neighbour's upper halo, and back
        assert {tr["to"]: tr["tag"] for tr in plan} == {"lower": 0, "upper": 1}
    with pytest.raises(ValueError):
        slab_halo_plan(0)


# --- blocks in several directions on CPU ranks --------------------------------------
# A 2 x 2 grid of blocks (z and t split) over four gloo ranks: each rank holds
# its block with one halo layer in z and t, flows it stage by stage with the
# oracle and exchanges faces on block_halo_plan's schedule (z, then t, faces
# carrying the z halos: the edges the staples and clover need).
BLK_N, BLK_SUB = (3, 2, 4, 6), (3, 2, 2, 3)


def _block_rank_main(rank, world, port, q):
    import sys

    import numpy as np

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist

    from latticeyangmills_b200 import block_halo_plan, block_layout
    from oracle import ymoracle as yo

    dist.init_process_group("gloo")
    n = BLK_N
    grid, blocks = block_layout(n, BLK_SUB)
    origin, extent = blocks[rank]
    split = [grid[d] > 1 for d in range(4)]
    local = [extent[d] + 2 * split[d] for d in range(4)]
    whole = yo.gen_expiah(n, 0.4, 13)  # (t, z, y, x, 4, 18)
    # the block with its halos, from the whole field (periodic)
    idx = [np.array([(origin[d] - split[d] + k) % n[d] for k in range(local[d])]) for d in range(4)]
    U = np.ascontiguousarray(whole[np.ix_(idx[3], idx[2], idx[1], idx[0])])
    Z = np.zeros_like(U)

    def layer(d, k):  # local coordinate k in direction d (numpy axis 3 - d)
        sl = [slice(None)] * 4
        sl[3 - d] = k
        return tuple(sl)

    plan = block_halo_plan(grid, rank, local)
    for _ in range(3):
        for stage in range(3):
            yo.flow_stage(U, Z, local, 0.02, stage)
            for ph, tr in enumerate(plan):
                d = tr["dir"]
                bufs, reqs = [], []
                for side, peer, send_k, recv_k, tag in (
                        ("lower", tr["lower"], tr["send_to_lower"], tr["recv_from_upper"], 2 * ph),
                        ("upper", tr["upper"], tr["send_to_upper"], tr["recv_from_lower"], 2 * ph + 1)):
                    reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(U[layer(d, send_k)])), peer,
                                           tag=tag))
                # what the upper neighbour sends down lands in the upper halo, and the other way round
                for peer, recv_k, tag in ((tr["upper"], tr["recv_from_upper"], 2 * ph),
                                          (tr["lower"], tr["recv_from_lower"], 2 * ph + 1)):
                    buf = torch.empty(U[layer(d, recv_k)].shape, dtype=torch.float64)
                    reqs.append(dist.irecv(buf, peer, tag=tag))
                    bufs.append((recv_k, buf))
                for r in reqs:
                    r.wait()
                for recv_k, buf in bufs:
                    U[layer(d, recv_k)] = buf.numpy()
    own = U[tuple(slice(split[d], split[d] + extent[d]) for d in (3, 2, 1, 0))].copy()
    parts = [None] * world
    dist.all_gather_object(parts, (origin, own))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        got = np.empty_like(whole)
        for o, part in parts:
            got[o[3]:o[3] + part.shape[0], o[2]:o[2] + part.shape[1], o[1]:o[1] + part.shape[2],
                o[0]:o[0] + part.shape[3]] = part
        want = whole.copy()
        for _ in range(3):
            yo.flow(want, n, 0.02, 1, 0)
        q.put(float(np.abs(got - want).max()))


def test_block_halo_exchange_in_two_directions_reproduces_the_whole_lattice_flow():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_block_rank_main, args=(r, 4, port, q)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    assert q.get(timeout=10) == 0.0  # bit for bit


def test_block_layout_and_plan():
    from latticeyangmills_b200 import block_halo_plan, block_layout

    grid, blocks = block_layout((8, 4, 6, 10), (4, 4, 3, 5))
    assert grid == [2, 1, 2, 2] and len(blocks) == 8
    assert blocks[1] == ((4, 0, 0, 0), (4, 4, 3, 5)) and blocks[2] == ((0, 0, 3, 0), (4, 4, 3, 5))
    plan = block_halo_plan(grid, 0, (6, 4, 5, 7))
    assert [tr["dir"] for tr in plan] == [0, 2, 3]
    assert [(tr["lower"], tr["upper"]) for tr in plan] == [(1, 1), (2, 2), (4, 4)]
    assert plan[2]["send_to_upper"] == 5 and plan[2]["recv_from_upper"] == 6
    with pytest.raises(ValueError):
        block_layout((8, 4, 6, 10), (3, 4, 3, 5))
