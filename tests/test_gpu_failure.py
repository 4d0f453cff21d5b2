"""Failure paths on a B200, without a GPU fault.

The product kernels wait on their operand copies with a time limit; when a wait runs out the
kernel sets an error word, stops issuing copies, waits (bounded) for the copies it already issued
and leaves, and the call returns BPMAX_ETIMEOUT. The test makes the waits run out the only safe
way: the one-shot test mode BPMAX_TUNE_INJECT_WAIT_TIMEOUT issues no copy at all, so nothing is in
flight when a wait gives up; the context must then give correct results on the next call.
"""
import numpy as np
import pytest

from bpmax_b200 import BpmaxError, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    yield e
    e.close()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("M,N", [(20, 40), (12, 64), (9, 16)])
def test_wait_timeout_is_reported_and_the_context_stays_usable(eng, oracle_mod, M, N):
    s1, s2 = W.pair(M, N, 300 + M)
    eng.set_weights(W.INTEGER_WEIGHTS)
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    default_limit = eng.get_tuning("wait_limit_us")
    try:
        eng.set_tuning("wait_limit_us", 2000)
        eng.set_tuning("inject_wait_timeout", 1)
        with pytest.raises(BpmaxError) as e:
            eng.score(s1, s2)
        assert e.value.status == 5  # BPMAX_ETIMEOUT
        assert eng.get_tuning("inject_wait_timeout") == 0  # one-shot
    finally:
        eng.set_tuning("wait_limit_us", default_limit)
    F, score = eng.fill_compact(s1, s2)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, M, N)


def test_wait_timeout_in_the_reference_layout_fill(eng, oracle_mod):
    M, N, T = 10, 24, 8
    s1, s2 = W.pair(M, N, 311)
    eng.set_weights(W.INTEGER_WEIGHTS)
    default_limit = eng.get_tuning("wait_limit_us")
    try:
        eng.set_tuning("wait_limit_us", 2000)
        eng.set_tuning("inject_wait_timeout", 1)
        with pytest.raises(BpmaxError) as e:
            eng.fill(s1, s2, T)
        assert e.value.status == 5
    finally:
        eng.set_tuning("wait_limit_us", default_limit)
    Fr, _ = eng.fill(s1, s2, T)
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert np.array_equal(bits(oracle_mod.to_reference_layout(Fo, M, N, T)[mask]), bits(Fr[mask]))


def test_wait_limit_validation(eng):
    with pytest.raises(BpmaxError):
        eng.set_tuning("wait_limit_us", 0)
    eng.set_tuning("wait_limit_us", 4_000_000)
    assert eng.get_tuning("wait_limit_us") == 4_000_000
