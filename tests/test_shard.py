"""Batch sharding across ranks (bpmax_b200.shard) on the CPU: the LPT partition's balance bound, and
two gloo ranks whose gathered scores equal the single-rank result. The per-rank scores come from
the oracle on tiny pairs (the GPU engine takes the oracle's place on a GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bpmax_b200 import shard, workloads as W


def test_lpt_partition_balance_and_cover():
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        costs = [int(x) for x in rng.integers(1, 10_000, size=97)]
        shares = shard.lpt_partition(costs, world)
        assert sorted(i for s in shares for i in s) == list(range(97))  # every pair exactly once
        loads = [sum(costs[i] for i in s) for s in shares]
        assert max(loads) - sum(costs) / world < max(costs)
    assert shard.lpt_partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert shard.lpt_partition([1, 2], 4) == [[1], [0], [], []]


def test_batch_shares_follow_padded_work():
    wl = W.batched_uneven(64, seed=4)
    shares = shard.shares_of(wl.pairs, 4)
    loads = [sum(shard.pair_cost(len(wl.pairs[i][0]), len(wl.pairs[i][1])) for i in s) for s in shares]
    assert max(loads) / min(loads) < 1.1
    assert shard.padded_width(9) == 16 and shard.padded_width(64) == 64 and shard.padded_width(65) == 128


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_scores(pairs):
    from oracle import oracle as O

    return np.array([O.score(O.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                    dtype=np.float32)


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.batched_uneven(11, seed=21, m_range=(1, 9), n_range=(1, 12))
        scores, mine = shard.run_sharded(_oracle_scores, wl.pairs, rank, world)
        out[rank] = (scores.tolist(), mine)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_single_rank_scores():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    wl = W.batched_uneven(11, seed=21, m_range=(1, 9), n_range=(1, 12))
    single, _ = shard.run_sharded(_oracle_scores, wl.pairs, 0, 1)
    assert res[0][0] == res[1][0] == single.tolist()       # every rank holds the whole batch's scores
    assert sorted(res[0][1] + res[1][1]) == list(range(11))  # the shares cover the batch once
    assert res[0][1] and res[1][1]
