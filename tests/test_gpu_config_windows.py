"""Configurations 2 (1024 x 64) and 3 (256 x 256, uniform and GC-rich) pinned bit for bit.

F(i1, j1, ., .) with j1 < K depends only on seq1[0..K) and seq2, and with i1 >= M-K only on
seq1[M-K..M) and seq2 (every candidate reads cells inside [i1, j1] x [i1, j1] and the single-strand
tables of the same ranges). So the oracle's fill of the prefix pair (seq1[:K], seq2) gives exactly
the cells j1 < K of the full-size table, and the fill of the suffix pair (seq1[M-K:], seq2) the cells
i1 >= M-K. Each case runs the full-size fill on the GPU (every outer diagonal, the multi-chunk
product jobs and the split schedule at full width), reads both windows back and compares them with
the oracle; it also fills the prefix pair itself on the GPU.
"""
import numpy as np
import pytest

from bpmax_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    yield e
    e.close()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("M,N,seed,gc,K", [
    (1024, 64, 2, False, 96),   # the default bench pair (configuration 2)
    (256, 256, 3, False, 20),   # configuration 3, uniform
    (256, 256, 3, True, 20),    # configuration 3, GC-rich (P(G) = P(C) = 0.35)
], ids=["cfg2_1024x64", "cfg3_256x256", "cfg3_256x256_gcrich"])
def test_full_size_windows_vs_oracle(eng, oracle_mod, M, N, seed, gc, K):
    wl = W.single_pair(M, N, seed, gc_rich=gc)
    s1, s2 = wl.pairs[0]
    eng.set_weights(wl.weights)
    eng.score(s1, s2)
    windows = {"prefix": (eng.read_cells(0, 0, K, 0, K, N), s1[:K]),
               "suffix": (eng.read_cells(0, M - K, M, M - K, M, N), s1[M - K:])}
    iu, ju = np.triu_indices(K)
    for name, (win, sub) in windows.items():
        Fo, _, _ = oracle_mod.fill(sub, s2, wl.weights)
        assert np.array_equal(bits(win[iu, ju]), bits(Fo)), name
        assert np.isnan(win[ju[ju != iu], iu[ju != iu]]).all()  # outer cells i1 > j1 are marked
    # the prefix pair on its own
    F, score = eng.fill_compact(s1[:K], s2)
    Fo, _, _ = oracle_mod.fill(s1[:K], s2, wl.weights)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, K, N)


def test_read_cells_rejects_bad_windows(eng):
    from bpmax_b200 import BpmaxError

    s1, s2 = W.pair(10, 12, 5)
    eng.score(s1, s2)
    for args in [(1, 0, 2, 0, 2), (0, 0, 11, 0, 2), (0, 3, 3, 0, 2), (0, -1, 2, 0, 2)]:
        with pytest.raises(BpmaxError):
            eng.read_cells(*args, 12)
    w = eng.read_cells(0, 2, 5, 4, 10, 12)
    assert w.shape == (3, 6, 12, 12)
