"""The window argument the full-size parity checks rest on, checked on the CPU.

F(i1, j1, ., .) with j1 < K depends only on seq1[0..K) and seq2, and with i1 >= M-K only on
seq1[M-K..M): the oracle's fill of the full pair equals its fills of the prefix and suffix pairs on
those cells, and bench.py's windowed comparison against the reference's own fill (driven here by an
engine stand-in that serves windows of the oracle's full table) finds no mismatch.
"""
import numpy as np
import pytest

import bench
from bpmax_b200 import workloads as W


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_prefix_and_suffix_windows_of_the_oracle(oracle_mod):
    M, N, K = 30, 19, 11
    s1, s2 = W.pair(M, N, 5)
    F, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    Fp, _, _ = oracle_mod.fill(s1[:K], s2, W.INTEGER_WEIGHTS)
    Fs, _, _ = oracle_mod.fill(s1[M - K:], s2, W.INTEGER_WEIGHTS)
    for a in range(K):
        for b in range(a, K):
            assert np.array_equal(bits(F[oracle_mod.cell(M, a, b)]), bits(Fp[oracle_mod.cell(K, a, b)]))
            lo = M - K
            assert np.array_equal(bits(F[oracle_mod.cell(M, lo + a, lo + b)]), bits(Fs[oracle_mod.cell(K, a, b)]))


class _OracleWindows:
    """Stands in for the engine's read_cells with windows of the oracle's table of one pair."""

    def __init__(self, oracle_mod, s1, s2, w):
        self.O = oracle_mod
        self.M, self.N = len(s1), len(s2)
        self.F, _, _ = oracle_mod.fill(s1, s2, w)

    def read_cells(self, pair, i_lo, i_hi, j_lo, j_hi, N):
        out = np.full((i_hi - i_lo, j_hi - j_lo, N, N), np.nan, dtype=np.float32)
        for a in range(i_lo, i_hi):
            for b in range(max(a, j_lo), j_hi):
                out[a - i_lo, b - j_lo] = self.F[self.O.cell(self.M, a, b)]
        return out


def test_bench_windows_against_the_reference(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("the reference's own fill was not built")
    M, N, T = 26, 20, 8
    wl = W.single_pair(M, N, seed=9)
    s1, s2 = wl.pairs[0]
    eng = _OracleWindows(oracle_mod, s1, s2, wl.weights)
    res = bench.windows_vs_reference(eng, wl, 9, 7, T)
    assert res["mismatches"] == 0 and res["cells"] > 0
    assert res["prefix"]["K"] == 9 and res["suffix"]["K"] == 7
    # a planted mistake in one window cell is found
    eng.F[oracle_mod.cell(M, M - 3, M - 1), 2, 5] += 1.0
    assert bench.windows_vs_reference(eng, wl, 9, 7, T)["suffix"]["mismatches"] == 1
