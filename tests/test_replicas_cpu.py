"""The multi-GPU form of this path is replicas (no exchange step): each rank
ranks its own panel and the job is timed by the slowest rank.  Two gloo ranks
on the CPU check the host logic bench.py uses for that -- the max-over-ranks
reduction, the barrier, and the whole-job throughput -- without a GPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        # rank r "took" 10 + r ms and an e2e time of 50 - r ms
        got = bench.max_over_ranks([10.0 + rank, 50.0 - rank], "cpu")
        dist.barrier()
        q.put((rank, got, bench.job_throughput(world, 1000, got[0])))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, value in out:
        assert got == [11.0, 50.0], (rank, got)
        assert value == pytest.approx(2 * 1000 / 11e-3 / 1e9)
