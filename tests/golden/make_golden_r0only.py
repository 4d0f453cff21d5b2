"""Generates tests/golden/r0only.npz from the REFERENCE's own R0-only program.

Run in a container that holds the reference sources (oracle/Makefile builds the program into
oracle/_ref/ospsqmax_check from IPDPSW/source/R0/ospsq_coarse_diag_top_down/src):

    make -C oracle && python tests/golden/make_golden_r0only.py

Each case: seeded non-negative integer sequences (small values, or rand()-sized values as the
reference's own driver draws them, IPDPSW/.../ospsqmax_float-wrapper.c, srand/rand), the
reference's F for every (i1 <= j1, i2 <= j2) in the compact layout, checked here against the
oracle restatement bit for bit. Small cases store the whole table, larger ones its SHA-256.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# name, M, N, seed, largest value (exclusive)
CASES = [
    ("r0_2x2", 2, 2, 201, 10),
    ("r0_5x7", 5, 7, 202, 50),
    ("r0_6x16_rand", 6, 16, 203, 2**31 - 1),
    ("r0_8x20", 8, 20, 204, 1000),
    ("r0_4x33_rand", 4, 33, 205, 2**31 - 1),
    ("r0_3x64", 3, 64, 206, 100),
    ("r0_5x70_rand", 5, 70, 207, 2**31 - 1),
    ("r0_2x130", 2, 130, 208, 1000),
]
FULL_MAX = 16000  # floats: store the table itself up to this size


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def main() -> None:
    out = {}
    for name, M, N, seed, hi in CASES:
        rng = np.random.default_rng(seed)
        s1 = rng.integers(0, hi, M).astype(np.int32)
        s2 = rng.integers(0, hi, N).astype(np.int32)
        F = O.ref_r0only(s1, s2)
        assert np.array_equal(F.view(np.uint32), O.r0only(s1, s2).view(np.uint32)), name
        out[f"{name}/seq1"] = s1
        out[f"{name}/seq2"] = s2
        out[f"{name}/sha"] = np.array(sha(F))
        if F.size <= FULL_MAX:
            out[f"{name}/F"] = F
        print(name, M, N, F.size, sha(F)[:12])
    np.savez_compressed(os.path.join(HERE, "r0only.npz"), **out)


if __name__ == "__main__":
    main()
