"""Generates tests/golden/*.json|npz from the REFERENCE's own programs.

Run in a container that holds the reference sources (oracle/Makefile builds them into
oracle/_ref/libbpmax_ref.so):

    make -C oracle && python tests/golden/make_golden.py

For every case it runs the reference's memoised verify program (bpmax_verify,
TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src/bpmax_verify.c:156) and, where the
reference accepts the tile parameters, its optimised fill (bpmax, V3/bpmax.c:129). It asserts
the two agree on every logical cell, then stores the sequences, weights, the score, SHA-256
digests of the logical table and of every reference-layout cell the fill writes, and (small
cases) the whole logical table. The reference has no golden vectors of its own: its tests use
clock-seeded rand() (V3/bpmax-wrapper.c:219), so these fixtures are the pinned known answers.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from bpmax_b200 import workloads as W  # noqa: E402

BASES = "ACGU"


def enc(s) -> str:
    return "".join(BASES[int(b)] for b in s)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


# name, M, N, N_tile, MR, NR (None: verify only), seed, weights, gc_rich, store_full
CASES = [
    ("tiny_1x8", 1, 8, None, None, None, 101, "integer", False, True),
    ("tiny_5x17_pad", 5, 17, 8, 1, 8, 102, "integer", False, True),
    ("tiny_6x12_pad", 6, 12, 8, 3, 8, 103, "integer", False, True),
    ("small_12x9_refw", 12, 9, 8, 3, 8, 104, "reference", False, True),
    ("small_9x24", 9, 24, 8, 2, 8, 105, "integer", False, True),
    ("small_16x16_realw", 16, 16, 8, 3, 8, 106, "random", False, True),
    ("ragged_37x23", 37, 23, 16, 3, 8, 107, "integer", False, False),
    ("ragged_29x41_realw", 29, 41, 24, 3, 24, 108, "random", False, False),
    ("gcrich_40x40", 40, 40, 16, 3, 8, 109, "integer", True, False),
    ("edge_64x8", 64, 8, None, None, None, 110, "integer", False, False),
    ("cfg_128x32", 128, 32, 16, 3, 8, 1, "integer", False, False),
]


def weights(kind: str, seed: int) -> np.ndarray:
    if kind == "integer":
        return W.INTEGER_WEIGHTS.copy()
    if kind == "reference":
        return W.REFERENCE_WEIGHTS.copy()
    return W.random_weights(seed)


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libbpmax_ref.so missing: run make -C oracle where the reference exists")
    index = []
    for name, M, N, T, MR, NR, seed, wk, gc, full in CASES:
        s1, s2 = W.pair(M, N, seed, W.GC_RICH if gc else None)
        w = weights(wk, seed)
        F4 = O.ref_verify(s1, s2, w)
        Fv = O.compact_from_4d(F4, M, N)
        rec = {
            "name": name, "M": M, "N": N, "seed": seed, "weights_kind": wk,
            "weights": [float(x) for x in w], "weights_hex": [float(x).hex() for x in w],
            "seq1": enc(s1), "seq2": enc(s2),
            "score": float(Fv[O.cell(M, 0, M - 1), 0, N - 1]),
            "logical_sha256": sha(Fv),
            "sources": ["bpmax_verify"],
        }
        if T is not None:
            Fr = O.ref_fill(s1, s2, w, T, MR, NR)
            Fl = O.logical_from_reference(Fr, M, N, T)
            assert np.array_equal(Fl.view(np.uint32), Fv.view(np.uint32)), name
            mask = O.reference_written_mask(M, N, T)
            assert not np.isnan(Fr[mask]).any() and np.isnan(Fr[~mask]).all(), name
            rec.update({"N_tile": T, "MR": MR, "NR": NR, "reference_layout_sha256": sha(Fr[mask]),
                        "reference_layout_floats": int(Fr.size)})
            rec["sources"].append("bpmax")
        if full:
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), F=Fv)
            rec["full_table"] = f"{name}.npz"
        index.append(rec)
        print(name, rec["score"], rec["sources"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generated_by": "tests/golden/make_golden.py", "cases": index}, f, indent=1)


if __name__ == "__main__":
    main()
