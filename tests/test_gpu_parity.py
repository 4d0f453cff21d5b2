"""CUDA fill vs the reference's golden fixtures and the oracle: bit-exact on every cell."""
import os
import subprocess

import numpy as np
import pytest

import golden_cases as G
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


@pytest.mark.parametrize("case", G.cases(), ids=lambda c: c["name"])
def test_golden_compact(eng, case):
    s1, s2, w = G.decode(case["seq1"]), G.decode(case["seq2"]), G.weights(case)
    eng.set_weights(w)
    F, score = eng.fill_compact(s1, s2)
    assert score == case["score"]
    assert G.sha(F) == case["logical_sha256"]
    full = G.full_table(case)
    if full is not None:
        assert np.array_equal(bits(full), bits(F))


@pytest.mark.parametrize("case", [c for c in G.cases() if "reference_layout_sha256" in c], ids=lambda c: c["name"])
def test_golden_reference_layout(eng, case, oracle_mod):
    s1, s2, w = G.decode(case["seq1"]), G.decode(case["seq2"]), G.weights(case)
    M, N, T = case["M"], case["N"], case["N_tile"]
    eng.set_weights(w)
    Fr, score = eng.fill(s1, s2, T)
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert score == case["score"]
    assert G.sha(Fr[mask]) == case["reference_layout_sha256"]
    # outer cells i1 > j1 are never touched (the caller's NaN fill survives)
    Ns = (N + T - 1) // T
    V = Fr.reshape(M, M, -1)
    lower = np.tril(np.ones((M, M), dtype=bool), -1)
    assert np.isnan(V[lower]).all()


@pytest.mark.parametrize("M,N,seed,wkind", [
    (1, 1, 1, "int"), (1, 5, 2, "int"), (3, 1, 3, "int"), (4, 4, 4, "int"), (2, 9, 5, "real"),
    (7, 8, 6, "int"), (13, 31, 7, "real"), (22, 33, 8, "int"), (17, 47, 9, "real"), (30, 64, 10, "int"),
    (9, 57, 11, "real"), (40, 17, 12, "int"), (5, 64, 13, "real"),
])
def test_random_vs_oracle(eng, oracle_mod, M, N, seed, wkind):
    s1, s2 = W.pair(M, N, seed)
    w = W.INTEGER_WEIGHTS if wkind == "int" else W.random_weights(seed)
    eng.set_weights(w)
    F, score = eng.fill_compact(s1, s2)
    Fo, _, _ = oracle_mod.fill(s1, s2, w)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, M, N)


def test_gc_rich_and_reference_weights(eng, oracle_mod):
    for (M, N, seed, gc, w) in [(26, 40, 21, True, W.INTEGER_WEIGHTS), (19, 24, 22, False, W.REFERENCE_WEIGHTS)]:
        s1, s2 = W.pair(M, N, seed, W.GC_RICH if gc else None)
        eng.set_weights(w)
        F, _ = eng.fill_compact(s1, s2)
        Fo, _, _ = oracle_mod.fill(s1, s2, w)
        assert np.array_equal(bits(F), bits(Fo))


def test_batched_uneven_matches_oracle_and_each(eng, oracle_mod):
    wl = W.batched_uneven(num_pairs=24, seed=77, m_range=(1, 40), n_range=(1, 64))
    eng.set_weights(wl.weights)
    got = eng.score_batch(wl.pairs)
    each = eng.score_each(wl.pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, wl.weights)[0], len(a), len(b)) for a, b in wl.pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(got), bits(exp))
    assert np.array_equal(bits(each), bits(exp))


def test_batched_bulk_finalize_matches_oracle(eng, oracle_mod):
    # 128 pairs of width class 64: the finalize launches of the first outer diagonals hold 2,048 or
    # more cells and take the 256-thread form, the later ones the 512-thread form
    rng = np.random.default_rng(91)
    pairs = [(W.random_sequence(20, rng), W.random_sequence(int(rng.integers(57, 65)), rng)) for _ in range(128)]
    eng.set_weights(W.INTEGER_WEIGHTS)
    got = eng.score_batch(pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(got), bits(exp))
    assert np.array_equal(bits(eng.score_each(pairs)), bits(exp))


def test_split_schedule_batch_of_one_width_class(eng, oracle_mod):
    """Several pairs of one width class (strand-2 lengths 57..64) take the split schedule: offset
    pair 0 of every cell is its own product launch and the other pairs run beside the finalize of
    the previous outer diagonal. M = 30 gives diagonals d >= 3, where the order of those launches
    matters; every score and one whole table must equal the oracle's."""
    rng = np.random.default_rng(93)
    pairs = [(W.random_sequence(30, rng), W.random_sequence(int(rng.integers(57, 65)), rng)) for _ in range(6)]
    eng.set_weights(W.INTEGER_WEIGHTS)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(eng.score_batch(pairs)), bits(exp))
    for p in (0, 5):
        win = eng.read_cells(p, 0, 30, 0, 30, len(pairs[p][1]))
        Fo, _, _ = oracle_mod.fill(*pairs[p], W.INTEGER_WEIGHTS)
        iu, ju = np.triu_indices(30)
        assert np.array_equal(bits(win[iu, ju]), bits(Fo))


def test_repeated_calls_and_shape_changes(eng, oracle_mod):
    eng.set_weights(W.INTEGER_WEIGHTS)
    for (M, N, seed) in [(12, 20, 31), (12, 20, 32), (6, 44, 33), (12, 20, 31)]:
        s1, s2 = W.pair(M, N, seed)
        assert eng.score(s1, s2) == oracle_mod.score(oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)[0], M, N)


def test_invalid_arguments_rejected(eng):
    from bpmax_b200 import BpmaxError

    with pytest.raises(BpmaxError):
        eng.score([0, 1, 5], [1, 2])
    with pytest.raises(BpmaxError):
        eng.set_weights([1.0] * 11 + [-1.0])
    with pytest.raises(BpmaxError):
        eng.fill([0, 1, 2], [1, 2, 3, 0, 1], 4)  # N < 8: the reference rejects it (V3/bpmax.c:131)
    # the context stays usable after an error
    eng.set_weights(W.INTEGER_WEIGHTS)
    assert eng.score([0, 1, 2, 3, 0, 2, 1, 3, 3], [3, 2, 1, 0, 2, 2]) >= 0


@pytest.mark.parametrize("M,N,seed,wkind", [
    (5, 65, 51, "int"), (7, 100, 52, "real"), (12, 130, 53, "int"), (3, 256, 54, "int"), (9, 200, 55, "real"),
    (16, 128, 56, "int"),
])
def test_wide_inner_tables_vs_oracle(eng, oracle_mod, M, N, seed, wkind):
    """Strand-2 lengths above 64 take the blocked product and the global-memory inner wavefront."""
    s1, s2 = W.pair(M, N, seed)
    w = W.INTEGER_WEIGHTS if wkind == "int" else W.random_weights(seed)
    eng.set_weights(w)
    F, score = eng.fill_compact(s1, s2)
    Fo, _, _ = oracle_mod.fill(s1, s2, w)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, M, N)


@pytest.mark.parametrize("M,N,seed,wkind", [(4, 330, 71, "int"), (3, 400, 72, "real"), (6, 343, 73, "int")])
def test_row_major_inner_tables_vs_oracle(eng, oracle_mod, M, N, seed, wkind):
    """Strand-2 lengths above 320 take the row-major tables: S2 by one launch per diagonal, the
    blocked product with its transposed copy, and the inner wavefront as one launch per inner
    diagonal over every cell of the outer diagonal."""
    s1, s2 = W.pair(M, N, seed)
    w = W.INTEGER_WEIGHTS if wkind == "int" else W.random_weights(seed)
    eng.set_weights(w)
    F, score = eng.fill_compact(s1, s2)
    Fo, _, _ = oracle_mod.fill(s1, s2, w)
    assert np.array_equal(bits(F), bits(Fo))
    assert score == oracle_mod.score(Fo, M, N)


def test_row_major_inner_tables_in_a_batch(eng, oracle_mod):
    pairs = [W.pair(m, n, 80 + i) for i, (m, n) in enumerate([(4, 330), (7, 40), (3, 352), (5, 100)])]
    eng.set_weights(W.INTEGER_WEIGHTS)
    got = eng.score_batch(pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(got), bits(exp))


def test_wide_inner_reference_layout(eng, oracle_mod):
    M, N, T = 6, 150, 64
    s1, s2 = W.pair(M, N, 57)
    eng.set_weights(W.INTEGER_WEIGHTS)
    Fr, _ = eng.fill(s1, s2, T)
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert np.array_equal(bits(oracle_mod.to_reference_layout(Fo, M, N, T)[mask]), bits(Fr[mask]))


def test_batched_mixed_widths(eng, oracle_mod):
    pairs = [W.pair(m, n, 60 + i) for i, (m, n) in enumerate([(9, 70), (14, 20), (5, 130), (11, 64), (8, 8), (3, 90)])]
    eng.set_weights(W.INTEGER_WEIGHTS)
    got = eng.score_batch(pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(got), bits(exp))


def test_tuning_settings_keep_results(eng, oracle_mod):
    """Every schedule setting changes how the work is cut, never a result bit."""
    pairs = [W.pair(m, n, 80 + i) for i, (m, n) in enumerate([(23, 61), (17, 30), (9, 12), (31, 64), (6, 45),
                                                                (7, 150), (5, 250)])]
    eng.set_weights(W.INTEGER_WEIGHTS)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, W.INTEGER_WEIGHTS)[0], len(a), len(b)) for a, b in pairs],
                   dtype=np.float32)
    keys = ("r0_pairs_per_job", "r0_merge_items", "class_streams", "r0_variant", "wide_stages", "class_share")
    saved = {k: eng.get_tuning(k) for k in keys}
    try:
        for ppj, merge, streams, variant, stages, share in [(1, 0, 1, 0, 2, 1), (3, 16, 0, 1, 3, 0),
                                                            (1 << 20, 2, 1, 1, 2, 1), (2, 1, 0, 0, 3, 0)]:
            eng.set_tuning("r0_pairs_per_job", ppj)
            eng.set_tuning("r0_merge_items", merge)
            eng.set_tuning("class_streams", streams)
            eng.set_tuning("r0_variant", variant)
            eng.set_tuning("wide_stages", stages)
            eng.set_tuning("class_share", share)
            assert np.array_equal(bits(eng.score_batch(pairs)), bits(exp))
            F, _ = eng.fill_compact(*pairs[0])
            Fo, _, _ = oracle_mod.fill(*pairs[0], W.INTEGER_WEIGHTS)
            assert np.array_equal(bits(F), bits(Fo))
    finally:
        for k, v in saved.items():
            eng.set_tuning(k, v)


def test_autotune_picks_a_setting_and_keeps_results(eng, oracle_mod):
    wl = W.batched_uneven(num_pairs=10, seed=79, m_range=(2, 28), n_range=(1, 64))
    wl.pairs += [W.pair(9, 140, 78), W.pair(6, 200, 77)]  # two tile-image widths
    eng.set_weights(wl.weights)
    before = eng.score_batch(wl.pairs)
    best, ms = eng.autotune(wl.pairs, trials=1)
    assert best["r0_pairs_per_job"] in (8, 32, 1 << 20) and best["r0_merge_items"] in (1, 4)
    assert best["class_streams"] in (0, 1) and best["r0_variant"] in (0, 1) and best["wide_stages"] in (2, 3)
    assert best["class_share"] in (0, 1)
    assert ms > 0
    after = eng.score_batch(wl.pairs)
    exp = np.array([oracle_mod.score(oracle_mod.fill(a, b, wl.weights)[0], len(a), len(b)) for a, b in wl.pairs],
                   dtype=np.float32)
    assert np.array_equal(bits(before), bits(exp)) and np.array_equal(bits(after), bits(exp))


def test_tuning_rejects_bad_values(eng):
    from bpmax_b200 import BpmaxError

    with pytest.raises(BpmaxError):
        eng.set_tuning("r0_pairs_per_job", 0)
    with pytest.raises(BpmaxError):
        eng._check(eng._L.bpmax_gpu_set_tuning(eng._ctx, 99, 1))


@pytest.mark.parametrize("case", [c for c in G.cases() if "reference_layout_sha256" in c][:3], ids=lambda c: c["name"])
def test_golden_reference_layout_pinned(eng, case, oracle_mod):
    """Into pinned host memory the table is copied out per outer diagonal (one strided copy each)
    instead of per row: same golden digest, the same NaN below the diagonal, and the same bytes as
    the pageable path."""
    import torch

    s1, s2, w = G.decode(case["seq1"]), G.decode(case["seq2"]), G.weights(case)
    M, N, T = case["M"], case["N"], case["N_tile"]
    eng.set_weights(w)
    n = eng.reference_size(M, N, T)
    buf = torch.full((n,), float("nan"), dtype=torch.float32, pin_memory=True)
    Fp, score = eng.fill(s1, s2, T, out=buf.numpy())
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert score == case["score"]
    assert G.sha(Fp[mask]) == case["reference_layout_sha256"]
    Fr, _ = eng.fill(s1, s2, T)
    assert np.array_equal(bits(Fp), bits(Fr))  # NaN patterns included


def test_reference_layout_pinned_vs_oracle(eng, oracle_mod):
    import torch

    M, N, T = 70, 64, 32
    s1, s2 = W.pair(M, N, 71)
    eng.set_weights(W.INTEGER_WEIGHTS)
    n = eng.reference_size(M, N, T)
    buf = torch.full((n,), float("nan"), dtype=torch.float32, pin_memory=True)
    Fp, _ = eng.fill(s1, s2, T, out=buf.numpy())
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert np.array_equal(bits(oracle_mod.to_reference_layout(Fo, M, N, T)[mask]), bits(Fp[mask]))
    lower = np.tril(np.ones((M, M), dtype=bool), -1)
    assert np.isnan(Fp.reshape(M, M, -1)[lower]).all()


def test_wide_reference_layout_pinned(eng, oracle_mod):
    """Pinned output with a strand-2 length over 64: one conversion launch and one strided copy per
    outer diagonal; the same bytes as the pageable path and the oracle's cells."""
    import torch

    M, N, T = 9, 150, 64
    s1, s2 = W.pair(M, N, 58)
    eng.set_weights(W.INTEGER_WEIGHTS)
    n = eng.reference_size(M, N, T)
    buf = torch.full((n,), float("nan"), dtype=torch.float32, pin_memory=True)
    Fp, _ = eng.fill(s1, s2, T, out=buf.numpy())
    Fr, _ = eng.fill(s1, s2, T)
    assert np.array_equal(bits(Fp), bits(Fr))
    Fo, _, _ = oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)
    mask = oracle_mod.reference_written_mask(M, N, T)
    assert np.array_equal(bits(oracle_mod.to_reference_layout(Fo, M, N, T)[mask]), bits(Fp[mask]))
