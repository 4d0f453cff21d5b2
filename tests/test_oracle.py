"""The oracle (CPU restatement of bpmax_verify.c) against the reference's golden fixtures and,
where the reference was built here, against the reference's own programs."""
import hashlib
import os

import numpy as np
import pytest

import golden_cases as G
from bpmax_b200 import workloads as W


@pytest.mark.parametrize("case", G.cases(), ids=lambda c: c["name"])
def test_oracle_matches_golden(oracle_mod, case):
    O = oracle_mod
    s1, s2, w = G.decode(case["seq1"]), G.decode(case["seq2"]), G.weights(case)
    M, N = case["M"], case["N"]
    F, S1, S2 = O.fill(s1, s2, w)
    assert O.score(F, M, N) == case["score"]
    assert G.sha(F) == case["logical_sha256"]
    full = G.full_table(case)
    if full is not None:
        assert np.array_equal(full.view(np.uint32), F.view(np.uint32))
    if "reference_layout_sha256" in case:
        T = case["N_tile"]
        mask = O.reference_written_mask(M, N, T)
        Fr = O.to_reference_layout(F, M, N, T)
        assert Fr.size == case["reference_layout_floats"]
        assert G.sha(Fr[mask]) == case["reference_layout_sha256"]


@pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).ref_available()")
@pytest.mark.parametrize("M,N,T,MR,NR,seed", [(7, 13, 8, 3, 8, 31), (11, 16, 8, 1, 8, 32), (4, 27, 24, 2, 24, 33)])
def test_oracle_matches_reference_programs(oracle_mod, M, N, T, MR, NR, seed):
    O = oracle_mod
    s1, s2 = W.pair(M, N, seed)
    w = W.random_weights(seed)
    F, _, _ = O.fill(s1, s2, w)
    Fv = O.compact_from_4d(O.ref_verify(s1, s2, w), M, N)
    assert np.array_equal(F.view(np.uint32), Fv.view(np.uint32))
    Fr = O.ref_fill(s1, s2, w, T, MR, NR, threads=2)
    mask = O.reference_written_mask(M, N, T)
    mine = O.to_reference_layout(F, M, N, T)
    assert np.array_equal(mine[mask].view(np.uint32), Fr[mask].view(np.uint32))


def test_oracle_rejects_bad_weights(oracle_mod):
    s1, s2 = W.pair(4, 8, 1)
    for bad in (-1.0, float("nan"), float("inf"), -0.0):
        w = W.INTEGER_WEIGHTS.copy()
        w[3] = bad
        with pytest.raises(ValueError):
            oracle_mod.fill(s1, s2, w)


def test_traceback_counts_sum_to_score_integer(oracle_mod):
    O = oracle_mod
    for seed in range(5):
        s1, s2 = W.pair(14, 11, 200 + seed)
        w = W.INTEGER_WEIGHTS
        F, S1, S2 = O.fill(s1, s2, w)
        c = O.traceback(s1, s2, w, F, S1, S2)
        assert np.all(c == np.round(c))
        assert float(c @ w.astype(np.float64)) == O.score(F, 14, 11)


def test_traceback_counts_match_finite_differences(oracle_mod):
    O = oracle_mod
    h = 1e-3
    checked = 0
    for seed in range(4):
        s1, s2 = W.pair(12, 10, 300 + seed)
        w = W.random_weights(300 + seed)
        F, S1, S2 = O.fill(s1, s2, w)
        c = O.traceback(s1, s2, w, F, S1, S2)
        assert abs(float(c @ w.astype(np.float64)) - O.score(F, 12, 10)) < 1e-3
        for t in range(12):
            wp, wm = w.copy(), w.copy()
            wp[t] += h
            wm[t] -= h
            fd = (O.score(O.fill(s1, s2, wp)[0], 12, 10) - O.score(O.fill(s1, s2, wm)[0], 12, 10)) / (2 * h)
            if abs(fd - c[t]) > 0.5:  # a tie or kink within h: FD is not a derivative there
                continue
            assert abs(fd - c[t]) < 0.05
            checked += 1
    assert checked >= 24


R0_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "r0only.npz")


def _r0_cases():
    z = np.load(R0_GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    return [(n, z[f"{n}/seq1"], z[f"{n}/seq2"], str(z[f"{n}/sha"]), z[f"{n}/F"] if f"{n}/F" in z.files else None)
            for n in names]


@pytest.mark.parametrize("case", _r0_cases(), ids=lambda c: c[0])
def test_r0only_oracle_matches_reference_golden(oracle_mod, case):
    """The R0-only restatement against tables the reference's own ospsqmax program printed."""
    name, s1, s2, digest, F = case
    got = oracle_mod.r0only(s1, s2)
    assert hashlib.sha256(got.tobytes()).hexdigest() == digest
    if F is not None:
        assert np.array_equal(got.view(np.uint32), F.view(np.uint32))


def test_r0only_oracle_matches_reference_program(oracle_mod):
    if not oracle_mod.ref_r0only_available():
        pytest.skip("the reference's R0-only program is not built here")
    rng = np.random.default_rng(17)
    for M, N in [(3, 5), (6, 9), (4, 17)]:
        s1, s2 = rng.integers(0, 2**31 - 1, M), rng.integers(0, 2**31 - 1, N)
        assert np.array_equal(oracle_mod.r0only(s1, s2).view(np.uint32), oracle_mod.ref_r0only(s1, s2).view(np.uint32))
