"""The persistent fill (BPMAX_TUNE_PERSISTENT): one launch per width class walks the outer diagonals
as a wavefront with device-side dependency counters instead of a graph of two launches per diagonal.
Every result must equal the oracle's bit for bit: single pairs of every width class, uneven batches
(several persistent launches side by side, or one after another), repeated calls, and the timeout
path (a wait that runs out ends the whole launch with BPMAX_ETIMEOUT and the context stays usable)."""
import numpy as np
import pytest

from bpmax_b200 import BpmaxError, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    e.set_tuning("persistent", 1)
    yield e
    e.close()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("M,N,seed,wkind", [
    (1, 1, 1, "int"), (2, 9, 2, "real"), (5, 8, 3, "int"), (13, 31, 4, "real"), (22, 33, 5, "int"),
    (30, 64, 6, "int"), (9, 57, 7, "real"), (40, 17, 8, "int"), (64, 48, 9, "real"), (37, 23, 10, "int"),
])
def test_persistent_single_pair_vs_oracle(eng, oracle_mod, M, N, seed, wkind):
    s1, s2 = W.pair(M, N, seed)
    w = W.INTEGER_WEIGHTS if wkind == "int" else W.random_weights(seed)
    eng.set_weights(w)
    F, score = eng.fill_compact(s1, s2)
    Fo, _, _ = oracle_mod.fill(s1, s2, w)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, M, N)


@pytest.mark.parametrize("mode", [1, 2])  # width classes side by side / one after another
def test_persistent_uneven_batch_vs_oracle(eng, oracle_mod, mode):
    wl = W.batched_uneven(num_pairs=40, seed=123, m_range=(1, 45), n_range=(1, 64))
    eng.set_weights(wl.weights)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, wl.weights)[0], len(a), len(b)) for a, b in wl.pairs],
                   dtype=np.float32)
    eng.set_tuning("persistent", mode)
    try:
        for _ in range(2):  # the second call replays the captured graph
            assert np.array_equal(bits(eng.score_batch(wl.pairs)), bits(exp))
        for p in (0, 7, 39):
            a, b = wl.pairs[p]
            win = eng.read_cells(p, 0, len(a), 0, len(a), len(b))
            Fo, _, _ = oracle_mod.fill(a, b, wl.weights)
            iu, ju = np.triu_indices(len(a))
            assert np.array_equal(bits(win[iu, ju]), bits(Fo))
    finally:
        eng.set_tuning("persistent", 1)


def test_persistent_batch_of_one_width_many_pairs(eng, oracle_mod):
    """Many pairs of one width class in one launch: product and finalize ranges span pairs."""
    rng = np.random.default_rng(9)
    pairs = [W.pair(int(rng.integers(1, 60)), 24, 300 + k) for k in range(30)]
    eng.set_weights(W.INTEGER_WEIGHTS)
    got = eng.score_batch(pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(got), bits(exp))
    for p in (0, 11, 29):
        a, b = pairs[p]
        win = eng.read_cells(p, 0, len(a), 0, len(a), len(b))
        Fo, _, _ = oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)
        iu, ju = np.triu_indices(len(a))
        assert np.array_equal(bits(win[iu, ju]), bits(Fo))


def test_persistent_large_pair_windows(eng, oracle_mod):
    """A 600 x 64 fill (long waits chains, many jobs per diagonal) against the oracle's prefix and
    suffix fills."""
    M, N, K = 600, 64, 48
    s1, s2 = W.pair(M, N, 77)
    eng.set_weights(W.INTEGER_WEIGHTS)
    eng.score(s1, s2)
    iu, ju = np.triu_indices(K)
    for lo, sub in ((0, s1[:K]), (M - K, s1[M - K:])):
        win = eng.read_cells(0, lo, lo + K, lo, lo + K, N)
        Fo, _, _ = oracle_mod.fill(sub, s2, W.INTEGER_WEIGHTS)
        assert np.array_equal(bits(win[iu, ju]), bits(Fo))


def test_persistent_matches_graph_path(eng, oracle_mod):
    wl = W.batched_uneven(num_pairs=16, seed=321, m_range=(20, 70), n_range=(8, 64))
    eng.set_weights(wl.weights)
    got = eng.score_batch(wl.pairs)
    eng.set_tuning("persistent", 0)
    try:
        ref = eng.score_batch(wl.pairs)
    finally:
        eng.set_tuning("persistent", 1)
    assert np.array_equal(bits(got), bits(ref))


def test_persistent_wait_timeout(eng, oracle_mod):
    M, N = 25, 40
    s1, s2 = W.pair(M, N, 55)
    eng.set_weights(W.INTEGER_WEIGHTS)
    default_limit = eng.get_tuning("wait_limit_us")
    try:
        eng.set_tuning("wait_limit_us", 2000)
        eng.set_tuning("inject_wait_timeout", 1)
        with pytest.raises(BpmaxError) as e:
            eng.score(s1, s2)
        assert e.value.status == 5
    finally:
        eng.set_tuning("wait_limit_us", default_limit)
    F, score = eng.fill_compact(s1, s2)
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    assert np.array_equal(bits(F), bits(Fo))
