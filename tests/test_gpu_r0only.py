"""R0-only double max-plus (bpmax_gpu_r0_only) against the reference's own R0-only program's
tables (tests/golden/r0only.npz) and the oracle: bit-exact on every cell."""
import hashlib
import os

import numpy as np
import pytest

from bpmax_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "r0only.npz")


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    yield e
    e.close()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _cases():
    z = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    return [(n, z[f"{n}/seq1"], z[f"{n}/seq2"], str(z[f"{n}/sha"])) for n in names]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_r0only_matches_reference_golden(eng, case):
    name, s1, s2, digest = case
    F, score = eng.r0_only(s1, s2)
    assert hashlib.sha256(F.tobytes()).hexdigest() == digest
    M, N = len(s1), len(s2)
    assert bits(np.float32(score)) == bits(F[M - 1, 0, N - 1])  # cell (0, M-1) is the M-th


@pytest.mark.parametrize("M,N,seed,hi", [(2, 9, 1, 100), (7, 9, 2, 2**31 - 1), (6, 40, 3, 1000), (5, 64, 4, 2**31 - 1),
                                         (9, 23, 5, 30), (4, 65, 6, 2**31 - 1), (3, 128, 7, 1000)])
def test_r0only_random_vs_oracle(eng, oracle_mod, M, N, seed, hi):
    rng = np.random.default_rng(seed)
    s1, s2 = rng.integers(0, hi, M), rng.integers(0, hi, N)
    F, _ = eng.r0_only(s1, s2)
    assert np.array_equal(bits(F), bits(oracle_mod.r0only(s1, s2)))


def test_r0only_then_fill_on_the_same_shape(eng, oracle_mod):
    """The context switches plans between the two modes and back."""
    s1, s2 = W.pair(6, 20, 9)
    eng.set_weights(W.INTEGER_WEIGHTS)
    F0, _ = eng.fill_compact(s1, s2)
    R, _ = eng.r0_only(s1, s2)
    F1, _ = eng.fill_compact(s1, s2)
    assert np.array_equal(bits(R), bits(oracle_mod.r0only(s1, s2)))
    assert np.array_equal(bits(F0), bits(F1))
    assert np.array_equal(bits(F1), bits(oracle_mod.fill(s1, s2, W.INTEGER_WEIGHTS)[0]))


def test_r0only_rejects_bad_arguments(eng):
    from bpmax_b200.api import BpmaxError

    with pytest.raises(BpmaxError):
        eng.r0_only([1, -2, 3], [4, 5, 6])
    with pytest.raises(BpmaxError):
        eng.r0_only([1], [4, 5, 6])
    F, _ = eng.r0_only([1, 2], [3, 4])  # still usable
    assert F[1, 0, 1] == 7.0  # F(0,1,0,1) = F(0,0,0,0) + F(1,1,1,1) = seq2[0] + seq2[1]
