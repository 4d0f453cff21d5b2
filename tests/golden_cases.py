"""Loads the golden fixtures generated from the reference (tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BASES = {"A": 0, "C": 1, "G": 2, "U": 3}


def cases():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)["cases"]


def decode(s: str) -> np.ndarray:
    return np.array([BASES[c] for c in s], dtype=np.int32)


def weights(case) -> np.ndarray:
    return np.array([float.fromhex(h) for h in case["weights_hex"]], dtype=np.float32)


def full_table(case):
    if "full_table" not in case:
        return None
    return np.load(os.path.join(GOLDEN, case["full_table"]))["F"]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()
