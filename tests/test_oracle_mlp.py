"""Pin the MLP gradient oracle itself: its analytic gradient equals a central
finite difference of its own loss (float64, bfloat16 rounding switched off so
that small perturbations are not rounded away)."""
import numpy as np


def test_mlp_oracle_gradient_matches_finite_difference(monkeypatch):
    from oracle import mlp
    monkeypatch.setattr(mlp, "bf16_round", lambda w: np.asarray(w, np.float64))
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp.NPARAM)
    X = rng.random((64, 8))
    T = rng.random(64)
    g, _ = mlp.gradients(p, X, T)
    for i in list(range(0, mlp.NPARAM, 97)) + [mlp.OFF_B3]:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.gradients(pp, X, T)[1] - mlp.gradients(pm, X, T)[1]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), i


def test_bf16_rounding_is_nearest_even():
    from oracle import mlp
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], np.float32)
    r = mlp.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                 # tie rounds to even
    assert r[2] == np.float32(1.0 + 2 ** -6)
    assert r[3] == -2.5
    assert np.isfinite(r[4])
