"""The replicas path of bench.py on CPU: two gloo ranks, each with its own
seeded batch, reduce to the slowest rank's time and the total work, and a
flag (parity, results equal) holds for the job only if it holds on every
rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    import datetime

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # each replica's own numbers: different times and batch sizes
    res = bench.reduce_over_ranks(dist, 1.0 + rank, 1000 * (rank + 1), 5e6 * (rank + 1), "cpu")
    flags = (bench.all_ranks_true(dist, True, "cpu"), bench.all_ranks_true(dist, rank == 0, "cpu"))
    out.put((rank, res + flags))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_reduce_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        elapsed, cands, cells, all_true, one_false = got[r]
        assert elapsed == pytest.approx(2.0)        # the slowest rank
        assert cands == pytest.approx(3000.0)       # all ranks' candidates
        assert cells == pytest.approx(1.5e7)
        assert all_true is True and one_false is False
