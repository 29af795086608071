"""CPU checks of the cost-model oracle itself: analytic gradients against
central finite differences, Adam against its closed form, feature sanity."""
import numpy as np

from oracle import sched_oracle as SO


def test_gradients_finite_difference():
    rng = np.random.default_rng(0)
    p = SO.init_params(1)
    X = rng.normal(size=(17, SO.N_FEAT))
    T = rng.normal(size=(17, SO.N_OUT))
    _, g = SO.loss_and_grads(p, X, T)
    eps = 1e-6
    for k in p:
        flat = p[k].reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + eps
            lp, _ = SO.loss_and_grads(p, X, T)
            flat[idx] = old - eps
            lm, _ = SO.loss_and_grads(p, X, T)
            flat[idx] = old
            num = (lp - lm) / (2 * eps)
            assert abs(num - g[k].reshape(-1)[idx]) <= 1e-6 + 1e-4 * abs(num), (k, idx)


def test_adam_first_step_is_signed_lr():
    p = {"w": np.array([1.0, -2.0, 3.0])}
    g = {"w": np.array([0.5, -0.1, 2.0])}
    m = {"w": np.zeros(3)}
    v = {"w": np.zeros(3)}
    SO.adam_step(p, g, m, v, 1, lr=0.01)
    np.testing.assert_allclose(p["w"], [1.0 - 0.01, -2.0 + 0.01, 3.0 - 0.01], atol=1e-7)


def test_features_sanity():
    from cuda_emd import workloads as W
    rng = np.random.default_rng(3)
    c = SO.trace_features(W.chirp_trace(rng, 4096))
    assert c[24] > 5 * c[17], "a rising chirp has denser extrema in its last eighth"
    assert abs(c[0] - 12 / 14) < 1e-12
    z = SO.trace_features(np.zeros(100))
    assert np.all(np.isfinite(z))
    assert z[29] == 1.0
