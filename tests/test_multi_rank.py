"""Multi-rank plumbing of bench.py on CPU: two gloo ranks, each filling its own independent pair
(weak scaling, no data-path collective), the step time taken as the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        wl = bench.workload("single", rank)
        s1, s2 = wl.pairs[0]
        bench.barrier(world, device="cpu")
        t = bench.reduce_max(world, 1.5 + rank, device="cpu")  # per-rank "device time"
        out[rank] = (len(s1), len(s2), int(s1[:64].sum()), t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_independent_pairs_and_max_time():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][:2] == res[1][:2] == (1024, 64)   # the same workload shape on every rank
    assert res[0][2] != res[1][2]                     # but its own sequences (independent pairs)
    assert res[0][3] == res[1][3] == 2.5              # every rank sees the max over ranks
