"""The N > 1 path of bench.py on CPU: two gloo ranks at 127.0.0.1 (no GPU).

With --gpus N every rank runs its own replica of the workload (replicas only, no data-path
collective); the only collectives are the barriers around the timed region and the max of
the ranks' times, and the reference arm runs on rank 0 alone.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        bench.barrier()
        t = bench.allmax(1.0 + rank)               # this rank's timed seconds
        value = bench.ns_per_day(100 * world, t)   # all ranks' steps over the slowest rank
        bench.barrier()

        class Args:
            steps, warmup, gpus = 3, 1, world

        ran = bench.run_reference(Args, rank) if rank != 0 else None   # rank > 0: no work
        out.put((rank, t, value, ran))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_the_max_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import bench
    for rank, t, value, ran in got:
        assert t == 2.0                                   # the slower rank's time on both
        assert value == pytest.approx(bench.ns_per_day(200, 2.0))
        assert ran is None
