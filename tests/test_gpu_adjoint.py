"""Adjoint pass (bpmax_gpu_grad_batch) vs the oracle's traceback with the reference tie-break,
and vs central finite differences of the GPU forward away from ties."""
import numpy as np
import pytest
import torch

from autograd_fn import BPMaxScore
from bpmax_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    yield e
    e.close()


def oracle_counts(O, pairs, w):
    out = []
    for a, b in pairs:
        F, S1, S2 = O.fill(a, b, w)
        out.append(O.traceback(a, b, w, F, S1, S2))
    return np.array(out)


@pytest.mark.parametrize("wkind", ["int", "ref", "real"])
def test_counts_match_oracle_traceback(eng, oracle_mod, wkind):
    rng = np.random.default_rng(7)
    pairs = [W.pair(int(rng.integers(1, 30)), int(rng.integers(1, 70)), 900 + i) for i in range(10)]
    w = {"int": W.INTEGER_WEIGHTS, "ref": W.REFERENCE_WEIGHTS, "real": W.random_weights(33)}[wkind]
    eng.set_weights(w)
    scores, grads = eng.grad_batch(pairs)
    exp = oracle_counts(oracle_mod, pairs, w)
    assert np.array_equal(grads.astype(np.float64), exp)
    exp_scores = np.array([oracle_mod.score(oracle_mod.fill(a, b, w)[0], len(a), len(b)) for a, b in pairs], np.float32)
    assert np.array_equal(scores.view(np.uint32), exp_scores.view(np.uint32))


def test_counts_wide_inner(eng, oracle_mod):
    pairs = [W.pair(7, 90, 950), W.pair(4, 130, 951)]
    w = W.random_weights(34)
    eng.set_weights(w)
    _, grads = eng.grad_batch(pairs)
    assert np.array_equal(grads.astype(np.float64), oracle_counts(oracle_mod, pairs, w))


def test_counts_match_finite_differences(eng):
    h = 1e-3
    pairs = [W.pair(20, 24, 960 + i) for i in range(4)]
    w = W.random_weights(35)
    eng.set_weights(w)
    scores, grads = eng.grad_batch(pairs)
    checked = 0
    for t in range(12):
        wp, wm = w.copy(), w.copy()
        wp[t] += h
        wm[t] -= h
        eng.set_weights(wp)
        sp = eng.score_batch(pairs).astype(np.float64)
        eng.set_weights(wm)
        sm = eng.score_batch(pairs).astype(np.float64)
        fd = (sp - sm) / (2 * h)
        ok = np.abs(fd - grads[:, t]) <= 0.5  # elsewhere a tie or kink lies within h
        assert np.all(np.abs(fd[ok] - grads[ok, t]) < 0.05)
        checked += int(ok.sum())
    assert checked >= 36


def test_autograd_function(eng):
    pairs = [W.pair(15, 18, 970), W.pair(9, 33, 971)]
    w = torch.tensor(W.random_weights(36), dtype=torch.float32, requires_grad=True)
    scores = BPMaxScore.apply(w, eng, pairs)
    scores.sum().backward()
    eng.set_weights(w.detach().numpy())
    _, grads = eng.grad_batch(pairs)
    assert torch.equal(w.grad, torch.from_numpy(grads.sum(axis=0)))
    # score = counts . w up to fp32 rounding of the sums
    assert torch.allclose(scores.double(), torch.from_numpy(grads).double() @ w.detach().double(), atol=1e-3)
