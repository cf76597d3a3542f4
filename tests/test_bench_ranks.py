"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, as torchrun starts them) combine their timed totals into the slowest
rank's, and the aggregate rate counts every rank's frames over that time."""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=30))
        r, w, loc = bench.dist_env()
        # rank k timed (1 + k) s on the device and (5 - k) s end to end
        tot = bench.reduce_max([1.0 + rank, 5.0 - rank], dist, "cpu")
        fps = bench.aggregate_fps(300, 5, w, tot[0])
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, (r, w, loc), tot, fps))
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None))


def test_two_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    got = sorted([q.get(timeout=120) for _ in procs])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, env, tot, fps in got:
        assert env != "error", tot
        assert env == (rank, 2, rank)
        assert tot == [2.0, 5.0]  # the slowest rank of each total
        assert fps == pytest.approx(300 * 5 * 2 / 2.0)


def test_single_rank_needs_no_group():
    import bench
    assert bench.reduce_max([1.5, 2.5], None, "cpu") == [1.5, 2.5]
    assert bench.aggregate_fps(300, 5, 1, 0.5) == pytest.approx(3000.0)
