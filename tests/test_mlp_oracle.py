"""Pins the surrogate network's oracle (oracle/mlp_ref.py) on the CPU: its back-propagated gradients
of the mean squared error equal central finite differences of its own FP64 loss, and its Adam step
and BF16 rounding follow their definitions. (The network has no counterpart in the reference, so
the oracle is pinned against the mathematics it restates.)"""
import numpy as np

from oracle import mlp_ref as R


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = (5, 8, 2, 7)  # n_in, hidden, n_hidden, n_out
    p = R.init_params(rng, *dims).astype(np.float64)
    p[-7:] = rng.normal(0, 0.3, 7)
    x = rng.standard_normal((6, 5))
    t = rng.standard_normal((6, 7))
    g, loss = R.gradients(p, x, t, *dims, emulate=False)
    # float32 parameters inside forward(): perturb in float32-representable steps
    idx = rng.choice(p.size, 40, replace=False)
    for i in idx:
        h = 1e-2
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = np.mean((R.forward(pp.astype(np.float32), x, *dims, emulate=False) - t) ** 2)
        lm = np.mean((R.forward(pm.astype(np.float32), x, *dims, emulate=False) - t) ** 2)
        fd = (lp - lm) / (np.float32(p[i] + h) - np.float32(p[i] - h))
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])) + 1e-5, (i, fd, g[i])


def test_adam_and_bf16_rounding():
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.1, -0.2, 0.0])
    pn, m, v = R.adam_step(p, g, np.zeros(3), np.zeros(3), 1, lr=0.01)
    # first step: update is lr * sign(g) (for |g| >> eps), none for g == 0
    assert np.allclose(pn - p, [-0.01, 0.01, 0.0], atol=1e-9)
    assert np.allclose(m, 0.1 * g) and np.allclose(v, 0.001 * g * g)
    # BF16: 8 significant bits, ties to even
    assert R.bf16(1.0 + 2 ** -8)[()] == 1.0            # tie -> even (1.0)
    assert R.bf16(1.0 + 3 * 2 ** -8)[()] == 1.0 + 2 ** -6  # tie -> even (upper)
    assert R.bf16(1.0 + 2 ** -7)[()] == 1.0 + 2 ** -7
    assert R.bf16(-3.14159)[()] == -3.140625
