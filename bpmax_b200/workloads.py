"""Seeded synthetic inputs and the named workloads of the BPMax fill.

Bases are encoded 0..3 = A,C,G,U (the reference's toNum mapping,
TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src/external_functions.c:70-85).
The reference itself draws ``rand() % 4`` seeded by the clock (V3/bpmax-wrapper.c:219-224); here
every sequence comes from a numpy PCG64 generator with an explicit seed so runs repeat.

Weights are a 12-entry table: intra-strand AU,UA,GC,CG,GU,UG then inter-strand AU,UA,GC,CG,GU,UG.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

PAIR_NAMES = ("AU", "UA", "GC", "CG", "GU", "UG")
WEIGHT_NAMES = tuple(f"intra_{p}" for p in PAIR_NAMES) + tuple(f"inter_{p}" for p in PAIR_NAMES)

#: The reference's hard-coded weights (V3/external_functions.c:58-68): AU=1.0, GC=3, GU=1.5.
REFERENCE_WEIGHTS = np.array([1.0, 1.0, 3.0, 3.0, 1.5, 1.5] * 2, dtype=np.float32)
#: Integer weights of the single-pair and batched workloads: GC=3, AU=2, GU=1 on both strands.
INTEGER_WEIGHTS = np.array([2.0, 2.0, 3.0, 3.0, 1.0, 1.0] * 2, dtype=np.float32)

GC_RICH = (0.15, 0.35, 0.35, 0.15)  # P(A), P(C), P(G), P(U)


def random_sequence(n: int, rng: np.random.Generator, probs=None) -> np.ndarray:
    if probs is None:
        return rng.integers(0, 4, size=n, dtype=np.int64).astype(np.int32)
    return rng.choice(4, size=n, p=np.asarray(probs, dtype=np.float64)).astype(np.int32)


def pair(m: int, n: int, seed: int, probs=None):
    """One (seq1, seq2) pair of lengths (m, n) from ``seed``."""
    rng = np.random.default_rng(seed)
    return random_sequence(m, rng, probs), random_sequence(n, rng, probs)


def random_weights(seed: int, lo: float = 0.5, hi: float = 4.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=12).astype(np.float32)


def terms(m: int, n: int) -> dict:
    """Max-plus candidate counts of one fill (one term = one fp32 add + one max).

    R0 = C(M)C(N); R1+R2 = 2 T(M) C(N); R3+R4 = 2 C(M) T(N); S1+S2 = C(M)+C(N), with
    C(n) = n(n^2-1)/6 and T(n) = n(n+1)/2. Twice the total is the reference's "bpmax OPS"."""
    C = lambda x: x * (x * x - 1) // 6
    T = lambda x: x * (x + 1) // 2
    r0 = C(m) * C(n)
    r12 = 2 * T(m) * C(n)
    r34 = 2 * C(m) * T(n)
    s = C(m) + C(n)
    return {"r0": r0, "r12": r12, "r34": r34, "s": s, "total": r0 + r12 + r34 + s}


@dataclass
class Workload:
    name: str
    pairs: list = field(default_factory=list)  # list of (seq1, seq2)
    weights: np.ndarray = field(default_factory=lambda: INTEGER_WEIGHTS.copy())

    @property
    def total_terms(self) -> int:
        return sum(terms(len(a), len(b))["total"] for a, b in self.pairs)


def single_pair(m: int, n: int, seed: int = 1, gc_rich: bool = False) -> Workload:
    s1, s2 = pair(m, n, seed, GC_RICH if gc_rich else None)
    tag = "gcrich" if gc_rich else "uniform"
    return Workload(f"single_{m}x{n}_{tag}", [(s1, s2)], INTEGER_WEIGHTS.copy())


def batched_uneven(num_pairs: int = 512, seed: int = 4, m_range=(16, 200), n_range=(8, 64)) -> Workload:
    """``num_pairs`` pairs, N1 ~ U[m_range], N2 ~ U[n_range] (inclusive), uniform ACGU."""
    rng = np.random.default_rng(seed)
    ps = []
    for _ in range(num_pairs):
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        ps.append((random_sequence(m, rng), random_sequence(n, rng)))
    return Workload(f"batched_{num_pairs}_uneven", ps, INTEGER_WEIGHTS.copy())


def gradient_batch(num_pairs: int = 64, m: int = 256, n: int = 64, seed: int = 5) -> Workload:
    """Pairs for the forward + adjoint workload with 12 random weights in [0.5, 4.0]."""
    rng = np.random.default_rng(seed)
    ps = [(random_sequence(m, rng), random_sequence(n, rng)) for _ in range(num_pairs)]
    return Workload(f"grad_{num_pairs}x{m}x{n}", ps, random_weights(seed + 1000))
