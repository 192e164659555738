"""The surrogate's GPU kernels (tensor-core forward/backward, Adam) against
the CPU oracle oracle/mlp_oracle.py, through the C ABI.

The oracle rounds to BF16 at the points the GPU stores BF16, so forward
values and gradients agree to FP32-accumulation error plus the occasional
one-ulp BF16 flip; the tolerances below are relative L2 errors per block.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("nang", [24, 365])
def test_forward_matches_oracle(nang):
    from smmp.surrogate import Surrogate
    s = Surrogate(nang, seed=11)
    p, norm = s.params()
    assert norm[0] == 0.0 and norm[1] == 1.0
    rng = np.random.default_rng(1)
    ang = rng.uniform(-np.pi, np.pi, (700, nang))
    got = s.predict(ang)
    want, _ = mo.forward(p, ang, s.nin_pad)
    assert _rel(got, want) < 5e-3
    # against the unrounded FP64 network: the BF16 storage error itself
    exact, _ = mo.forward(p, ang, s.nin_pad, round_bf16=False)
    assert _rel(got, exact) < 5e-2


@pytest.mark.parametrize("nang,B", [(24, 300), (365, 130)])
def test_gradients_match_oracle(nang, B):
    from smmp.surrogate import Surrogate
    s = Surrogate(nang, seed=5)
    p, _ = s.params()
    rng = np.random.default_rng(2)
    # random biases too, so every block's gradient is exercised
    lay = s.layout()
    for k in ("b1", "b2", "b3", "b4"):
        p[lay[k][0]] = rng.normal(0, 0.1, lay[k][0].stop - lay[k][0].start)
    s.set_params(p, np.array([0.0, 1.0], dtype=np.float32))
    ang = rng.uniform(-np.pi, np.pi, (B, nang))
    e = rng.normal(0, 1, B)
    loss, g = s.gradients(ang, e)
    wl, wg = mo.loss_and_grad(p, ang, e, s.nin_pad)
    assert loss == pytest.approx(wl, rel=1e-3)
    for k, (sl, _) in lay.items():
        assert _rel(g[sl], wg[sl]) < 2e-2, k


def test_training_fits_a_smooth_landscape():
    """Adam on a synthetic energy of 24 dihedrals: the held-out error falls
    well below the spread of the energies."""
    from smmp.surrogate import Surrogate
    rng = np.random.default_rng(3)
    nang, n = 24, 24000
    a, b = rng.normal(0, 2, nang), rng.normal(0, 1, nang)

    def energy(t):
        return (np.cos(t) @ a + np.sin(2 * t) @ b + 0.5 * np.cos(t[:, 0] - t[:, 1]) * 5)

    ang = rng.uniform(-np.pi, np.pi, (n, nang))
    e = energy(ang)
    s = Surrogate(nang, seed=9)
    s.set_data(ang[:20000], e[:20000])
    first = s.train(1, batch=256, lr=1e-3)
    last = s.train(14, batch=256, lr=1e-3)
    assert last < 0.2 * first
    pred = s.predict(ang[20000:])
    rmse = float(np.sqrt(np.mean((pred - e[20000:]) ** 2)))
    assert rmse < 0.15 * float(np.std(e)), (rmse, np.std(e))
