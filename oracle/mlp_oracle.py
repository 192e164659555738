"""CPU oracle of the energy surrogate's forward and backward passes (test
infrastructure only; the surrogate has no counterpart in the reference).

FP64 numpy restatement of the network the GPU trains: features sin/cos of
the free dihedrals, three hidden layers of 256 with SiLU, a linear output,
mean squared error.  With bf16=True the values the GPU stores in BF16 (inputs,
weights, hidden activations, hidden-layer gradients) are rounded to BF16 at
the same points, so the GPU's gradients can be compared element by element;
with bf16=False it is the exact FP64 network, which the finite-difference
test checks.

Parameter layout (flat FP32 vector): W1[nin_pad][256] b1 W2[256][256] b2
W3[256][256] b3 w4[256] b4.
"""
import numpy as np

H = 256


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def layout(nin_pad):
    sizes = [("W1", (nin_pad, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
             ("W3", (H, H)), ("b3", (H,)), ("w4", (H,)), ("b4", (1,))]
    out, off = {}, 0
    for name, shape in sizes:
        n = int(np.prod(shape))
        out[name] = (slice(off, off + n), shape)
        off += n
    return out, off


def unpack(p, nin_pad):
    lay, n = layout(nin_pad)
    assert p.size == n
    return {k: np.asarray(p[s], dtype=np.float64).reshape(shape) for k, (s, shape) in lay.items()}


def sigm(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * sigm(z)


def dsilu(z):
    s = sigm(z)
    return s * (1.0 + z * (1.0 - s))


def features(ang, nin_pad, round_bf16):
    a = np.asarray(ang, dtype=np.float32 if round_bf16 else np.float64)
    n, k = a.shape
    X = np.zeros((n, nin_pad))
    X[:, 0:2 * k:2] = np.sin(a)
    X[:, 1:2 * k:2] = np.cos(a)
    return bf16(X) if round_bf16 else X


def forward(p, ang, nin_pad, round_bf16=True):
    """Returns (y, cache) with y the network output (normalised units)."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    w = unpack(p, nin_pad)
    W1, W2, W3, w4 = r(w["W1"]), r(w["W2"]), r(w["W3"]), r(w["w4"])
    X = features(ang, nin_pad, round_bf16)
    Z1 = X @ W1 + w["b1"]
    H1 = r(silu(Z1))
    Z2 = H1 @ W2 + w["b2"]
    H2 = r(silu(Z2))
    Z3 = H2 @ W3 + w["b3"]
    H3 = r(silu(Z3))
    y = H3 @ w4 + w["b4"][0]
    return y, dict(X=X, Z1=Z1, H1=H1, Z2=Z2, H2=H2, Z3=Z3, H3=H3, W2=W2, W3=W3, w4=w4)


def loss_and_grad(p, ang, target, nin_pad, round_bf16=True):
    """Mean squared error of the batch and its gradient (flat, FP64)."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    y, c = forward(p, ang, nin_pad, round_bf16)
    B = y.shape[0]
    d = y - np.asarray(target, dtype=np.float64)
    loss = float(np.mean(d * d))
    dy = 2.0 * d / B
    dZ3 = r(dy[:, None] * c["w4"][None, :] * dsilu(c["Z3"]))
    g = {}
    g["w4"] = c["H3"].T @ dy
    g["b4"] = np.array([dy.sum()])
    g["W3"] = c["H2"].T @ dZ3
    g["b3"] = dZ3.sum(0)
    dZ2 = r((dZ3 @ c["W3"].T) * dsilu(c["Z2"]))
    g["W2"] = c["H1"].T @ dZ2
    g["b2"] = dZ2.sum(0)
    dZ1 = r((dZ2 @ c["W2"].T) * dsilu(c["Z1"]))
    g["W1"] = c["X"].T @ dZ1
    g["b1"] = dZ1.sum(0)
    lay, n = layout(nin_pad)
    flat = np.zeros(n)
    for k, (s, shape) in lay.items():
        flat[s] = g[k].reshape(-1)
    return loss, flat
