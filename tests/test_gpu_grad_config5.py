"""Configuration 5 at its stated shape: 64 pairs with N1 = 256, N2 = 64, uniform ACGU, and 12 weights
drawn from U[0.5, 4.0]. The adjoint pass returns d(score)/d(weights) as exact integer counts of the
optimal structure's pair types. Checked
* against central finite differences (h = 1e-3) of the GPU's own forward scores on 4 of the pairs:
  a (pair, weight) entry whose difference quotient lies more than 0.5 from the count sits at a tie or
  kink of the piecewise-linear score and is skipped; every other entry must agree to fp32 rounding,
  and most entries must be of that kind;
* against the oracle's traceback (the reference's tie-break; the reference itself has none) on the
  48-long strand-1 prefixes of the same pairs, where the CPU oracle finishes in seconds.
"""
import numpy as np
import pytest

from bpmax_b200 import workloads as W

pytestmark = pytest.mark.gpu

FD_TOL = 0.25  # fp32 rounding of two scores of a few hundred, divided by 2h


@pytest.fixture(scope="module")
def eng():
    from bpmax_b200 import Engine

    e = Engine(0)
    yield e
    e.close()


def test_config5_forward_and_adjoint(eng):
    wl = W.gradient_batch(64, 256, 64, seed=5)
    w = wl.weights
    eng.set_weights(w)
    scores, grads = eng.grad_batch(wl.pairs)
    assert grads.shape == (64, 12)
    assert np.array_equal(grads, np.round(grads)) and (grads >= 0).all()
    assert np.array_equal(scores.view(np.uint32), eng.score_batch(wl.pairs).view(np.uint32))
    # the optimum's value is its pair-type counts times the weights, up to fp32 rounding
    assert np.allclose(grads.astype(np.float64) @ w.astype(np.float64), scores, rtol=1e-5, atol=1e-3)
    sub = wl.pairs[:4]
    matched = 0
    for t in range(12):
        wp, wm = w.copy(), w.copy()
        wp[t] = np.float32(w[t] + np.float32(1e-3))
        wm[t] = np.float32(w[t] - np.float32(1e-3))
        eng.set_weights(wp)
        sp = eng.score_batch(sub).astype(np.float64)
        eng.set_weights(wm)
        sm = eng.score_batch(sub).astype(np.float64)
        fd = (sp - sm) / (np.float64(wp[t]) - np.float64(wm[t]))
        for p in range(4):
            err = abs(fd[p] - grads[p, t])
            if err > 0.5:
                continue  # tie or kink
            assert err < FD_TOL, (p, t, fd[p], grads[p, t])
            matched += 1
    assert matched >= 0.8 * 48, matched
    eng.set_weights(w)


def test_config5_counts_vs_oracle_traceback_on_prefixes(eng, oracle_mod):
    wl = W.gradient_batch(64, 256, 64, seed=5)
    pre = [(a[:48], b) for a, b in wl.pairs[:4]]
    eng.set_weights(wl.weights)
    scores, grads = eng.grad_batch(pre)
    for p, (a, b) in enumerate(pre):
        F, S1, S2 = oracle_mod.fill(a, b, wl.weights)
        assert scores[p] == oracle_mod.score(F, len(a), len(b))
        assert np.array_equal(grads[p].astype(np.float64), oracle_mod.traceback(a, b, wl.weights, F, S1, S2)), p
