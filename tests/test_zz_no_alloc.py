"""bpmax_gpu_score_noalloc: the entry point for callers that cannot allocate device memory.

Such callers (code inside another framework's memory pool or under a fixed device-memory budget,
and latency-critical code that must not risk the synchronisation cudaMalloc may imply) get a
score computed entirely in the library's fixed 64 MiB device scratch array. Its result must equal
the ordinary entry point's and the oracle's bit for bit, also on the second of two calls in a row
(the scratch keeps the previous call's contents), and repeated calls must not take device memory.
This file is collected last on purpose.
"""
import numpy as np
import pytest

from bpmax_b200 import api, workloads as W

pytestmark = pytest.mark.gpu

CASES = [(60, 61, 11, W.random_weights(11)),  # larger first: leaves stale tables behind
         (33, 29, 12, W.INTEGER_WEIGHTS)]


def bits(x):
    return np.float32(x).view(np.uint32)


def test_noalloc_matches_score_and_oracle_on_two_calls_in_a_row(oracle_mod):
    eng = api.Engine(0)
    try:
        expected = []
        for M, N, seed, w in CASES:
            s1, s2 = W.pair(M, N, seed)
            eng.set_weights(w)
            expected.append(eng.score(s1, s2))
    finally:
        eng.close()
    for (M, N, seed, w), exp in zip(CASES, expected):
        s1, s2 = W.pair(M, N, seed)
        got = api.score_noalloc(s1, s2, w)
        Fo, _, _ = oracle_mod.fill(s1, s2, w)
        assert bits(got) == bits(exp), (M, N, got, exp)
        assert bits(got) == bits(oracle_mod.score(Fo, M, N))


def test_noalloc_takes_no_device_memory():
    import torch

    pairs = [(W.pair(M, N, seed), w) for M, N, seed, w in CASES]
    for (s1, s2), w in pairs:  # first calls: the array's set-up and the kernels' first loads
        api.score_noalloc(s1, s2, w)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    scores = [[api.score_noalloc(s1, s2, w) for (s1, s2), w in pairs] for _ in range(3)]
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free0, (free0, free1)
    assert all(r == scores[0] for r in scores)


def test_noalloc_size_limit_is_an_error():
    s1, s2 = W.pair(115, 64, 13)  # T(115)*10080 bytes of tables + S1 + job lists > 64 MiB
    with pytest.raises(api.BpmaxError) as e:
        api.score_noalloc(s1, s2, W.INTEGER_WEIGHTS)
    assert e.value.status == 1
    s1, s2 = W.pair(114, 64, 14)  # the largest M that fits at N=64
    assert api.score_noalloc(s1, s2, W.INTEGER_WEIGHTS) > 0
