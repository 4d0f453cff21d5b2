"""bpmax_gpu_score_noalloc: the entry point for callers that cannot allocate device memory.

Such callers (code inside another framework's memory pool or under a fixed device-memory budget,
and latency-critical code that must not risk the synchronisation cudaMalloc may imply) get a
score computed entirely in the library's fixed 64 MiB device scratch array. Its result must equal
the ordinary entry point's bit for bit, also on the second of two calls in a row (the scratch keeps
the previous call's contents). This file is collected last on purpose.
"""
import numpy as np
import pytest

from bpmax_b200 import api, workloads as W

pytestmark = pytest.mark.gpu


def bits(x):
    return np.float32(x).view(np.uint32)


def test_noalloc_matches_score_on_two_calls_in_a_row():
    eng = api.Engine(0)
    try:
        cases = [(60, 61, 11, W.random_weights(11)),  # larger first: leaves stale tables behind
                 (33, 29, 12, W.INTEGER_WEIGHTS)]
        for M, N, seed, w in cases:
            s1, s2 = W.pair(M, N, seed)
            eng.set_weights(w)
            expected = eng.score(s1, s2)
            got = api.score_noalloc(s1, s2, w)
            assert bits(got) == bits(expected), (M, N, got, expected)
    finally:
        eng.close()


def test_noalloc_size_limit_is_an_error():
    s1, s2 = W.pair(115, 64, 13)  # T(115)*10080 bytes of tables + S1 + job lists > 64 MiB
    with pytest.raises(api.BpmaxError) as e:
        api.score_noalloc(s1, s2, W.INTEGER_WEIGHTS)
    assert e.value.status == 1
    s1, s2 = W.pair(114, 64, 14)  # the largest M that fits at N=64
    assert api.score_noalloc(s1, s2, W.INTEGER_WEIGHTS) > 0
