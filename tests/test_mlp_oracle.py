"""The surrogate's CPU oracle (oracle/mlp_oracle.py) against finite
differences, in exact FP64 (no BF16 rounding): its backward pass is the
reference the GPU gradients are checked against."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, -3.14159, 0.0])
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[4] == 0.0
    assert r[1] == 1.0                      # tie to even
    assert r[2] == 1.0 + 2.0 ** -7          # rounds up
    assert abs(r[3] + 3.140625) < 1e-12


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    nang, nin_pad, B = 5, 16, 12
    lay, n = mo.layout(nin_pad)
    p = rng.normal(0, 0.1, n)
    p[lay["W1"][0]] = rng.normal(0, 0.4, nin_pad * 256)
    ang = rng.uniform(-np.pi, np.pi, (B, nang))
    t = rng.normal(0, 1, B)
    loss, g = mo.loss_and_grad(p, ang, t, nin_pad, round_bf16=False)
    # padded input rows of W1 see zero features: zero gradient
    w1 = g[lay["W1"][0]].reshape(nin_pad, 256)
    assert np.all(w1[2 * nang:] == 0.0)
    idx = np.concatenate([rng.choice(np.arange(n)[lay[k][0]], 6, replace=False)
                          for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4")] +
                         [np.arange(n)[lay["b4"][0]]])
    idx = [i for i in idx if not (lay["W1"][0].start <= i < lay["W1"][0].stop
                                  and (i - lay["W1"][0].start) // 256 >= 2 * nang)]
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = mo.loss_and_grad(q, ang, t, nin_pad, round_bf16=False)
        q[i] -= 2 * h
        lm, _ = mo.loss_and_grad(q, ang, t, nin_pad, round_bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
