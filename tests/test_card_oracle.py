"""The estimator network's CPU oracle pinned on its own: its analytic gradient against
central finite differences of its loss (float64 parameters), and BF16 rounding against
values whose nearest BF16 neighbours are known."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.1, mlp.N_PARAMS)
    x = rng.normal(0, 1, (7, mlp.N_IN))
    t = rng.normal(0, 1, (7, mlp.N_OUT))
    m = (rng.random((7, mlp.N_OUT)) < 0.7).astype(np.float64)
    _, g = mlp.loss_and_grad(p, x, t, m, bf16=False)
    for i in rng.choice(mlp.N_PARAMS, 80, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        lp, _ = mlp.loss_and_grad(p + e, x, t, m, bf16=False)
        lm, _ = mlp.loss_and_grad(p - e, x, t, m, bf16=False)
        num = (lp - lm) / 2e-6
        assert abs(num - g[i]) <= 1e-7 + 1e-4 * abs(num), (i, num, g[i])


def test_bf16_forward_uses_rounded_weights():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.1, mlp.N_PARAMS).astype(np.float32)
    x = rng.normal(0, 1, (5, mlp.N_IN))
    q = p.copy()
    o = 0
    for s in mlp.SHAPES:
        n = int(np.prod(s))
        if len(s) == 2:
            q[o:o + n] = mlp.bf16_round(p[o:o + n])
        o += n
    y1, _ = mlp.forward(p, x, bf16=True)
    y2, _ = mlp.forward(q.astype(np.float64), x, bf16=False)
    np.testing.assert_allclose(y1, y2, rtol=1e-12, atol=1e-12)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -8 + 2 ** -20], np.float32)
    r = mlp.bf16_round(v)
    # ties go to the even neighbour; above the tie rounds up
    np.testing.assert_array_equal(r, np.array([1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6, -2.5, 1.0 + 2 ** -7],
                                              np.float32))
