"""Host side of the learned opening criterion: the numpy restatement of the
MLP gradient against finite differences, and the C ABI's model objects and
options (no kernel runs here)."""
import numpy as np
import pytest

from fastlinkingnumbers_b200 import FlnError, LearnedCriterion, learned_options
from fastlinkingnumbers_b200 import _native as N
from mlp_ref import B1, B3, W3, _features, _init, mlp_loss_grad


def test_numpy_gradient_matches_finite_differences():
    # Pins the restatement the GPU tests compare the training kernel with.
    rng = np.random.default_rng(0)
    p = _init(rng).astype(np.float64)
    X, T = _features(rng, 64), rng.uniform(-8, -2, 64).astype(np.float32)
    _, g = mlp_loss_grad(p, X, T, 0.9)
    for k in list(rng.integers(0, N.MLP_PARAMS, 40)) + [B3, W3 + 5, B1 + 3]:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (mlp_loss_grad(pp, X, T, 0.9)[0] - mlp_loss_grad(pm, X, T, 0.9)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(g[k]), k




def test_model_roundtrip_and_checks():
    p = _init(np.random.default_rng(3))
    m = LearnedCriterion.from_params(p, s_min=1.25, log10_tau=-5.5, min_candidates=6)
    np.testing.assert_array_equal(m.params(), p)
    info = m.info()
    assert (info["s_min"], info["log10_tau"], info["min_candidates"]) == (1.25, -5.5, 6)
    bad = p.copy()
    bad[7] = np.nan
    with pytest.raises(FlnError):
        LearnedCriterion.from_params(bad, s_min=1.0, log10_tau=-5.0)
    with pytest.raises(FlnError):
        LearnedCriterion.from_params(p, s_min=0.0, log10_tau=-5.0)


def test_default_options():
    o = learned_options()
    assert (o.s_min, o.sample_keep, o.epochs, o.batch, o.quantile, o.tau_quantile) == (1.5, 0.05, 40, 4096, 0.9, 0.5)
    assert (o.max_samples, o.max_terms, o.min_candidates, o.seed) == (1 << 20, 1 << 16, 4, 1)
    with pytest.raises(FlnError):
        learned_options(no_such_option=1)
