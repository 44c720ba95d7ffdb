"""CPU oracle of the learned-curvature network (test infrastructure only).

A numpy restatement of the forward and backward pass that the tensor-core
kernels (icls-release_b200/csrc/k_mlp.cu) compute, with the same rounding
points: each FP32 input enters as a BF16 pair hi = bf16(x), lo = bf16(x - hi);
the weights W1..W3, the hidden activations and the back-propagated deltas
are rounded to BF16 (round to nearest even) where the kernels feed them to a
BF16 tile; biases, W4, pre-activations, the head and every accumulation stay
in higher precision (float64 here, FP32 on the GPU).  The output is the
correction to the plain stencil's kappa * dx.
The network has no counterpart in the reference: it replaces the
get_curvature stencil of interface.f90:20-119 in the learned form.

Parameter layout (29057 floats): W1 [128][32], b1 [128], W2 [128][128],
b2 [128], W3 [64][128], b3 [64], W4 [64], b4.
"""
import numpy as np

IN, H1, H2, H3 = 32, 128, 128, 64
OFF = {}
_o = 0
for _name, _n in (("W1", H1 * IN), ("b1", H1), ("W2", H2 * H1), ("b2", H2), ("W3", H3 * H2), ("b3", H3),
                  ("W4", H3), ("b4", 1)):
    OFF[_name] = (_o, _o + _n)
    _o += _n
NPARAMS = _o


def bf16(x):
    """round float values to the nearest BF16 (ties to even), as float64"""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta):
    t = np.asarray(theta, dtype=np.float64)
    g = lambda n: t[OFF[n][0]:OFF[n][1]]
    return (g("W1").reshape(H1, IN), g("b1"), g("W2").reshape(H2, H1), g("b2"), g("W3").reshape(H3, H2), g("b3"),
            g("W4"), g("b4")[0])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(theta, X):
    """y of FP32 inputs X [n][32] and the pre-activations"""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(theta)
    X32 = np.asarray(X, dtype=np.float32)
    hi = bf16(X32)
    lo = bf16(X32 - hi.astype(np.float32))
    x = hi + lo  # both halves act through the same BF16 W1
    z1 = hi @ bf16(W1).T + lo @ bf16(W1).T + b1
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(W2).T + b2
    h2 = bf16(silu(z2))
    z3 = h2 @ bf16(W3).T + b3
    y = silu(z3) @ W4 + b4
    return y, (x, z1, h1, z2, h2, z3)


def gradient(theta, X, label, scale):
    """gradient of scale * sum (y - label)^2 / 2 ... as the kernels form it:
    dy = scale * (y - label) per sample; returns (grad[NPARAMS], sum e^2)"""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(theta)
    y, (x, z1, h1, z2, h2, z3) = forward(theta, X)
    e = y - np.asarray(label, dtype=np.float64)
    dy = scale * e
    g = np.zeros(NPARAMS)
    g[OFF["b4"][0]] = dy.sum()
    g[OFF["W4"][0]:OFF["W4"][1]] = silu(z3).T @ dy
    d3 = dy[:, None] * W4[None, :] * dsilu(z3)
    g[OFF["b3"][0]:OFF["b3"][1]] = d3.sum(axis=0)
    d3b = bf16(d3)
    g[OFF["W3"][0]:OFF["W3"][1]] = (d3b.T @ h2).ravel()
    dh2 = d3b @ bf16(W3)
    d2 = dh2 * dsilu(z2)
    g[OFF["b2"][0]:OFF["b2"][1]] = d2.sum(axis=0)
    d2b = bf16(d2)
    g[OFF["W2"][0]:OFF["W2"][1]] = (d2b.T @ h1).ravel()
    dh1 = d2b @ bf16(W2)
    d1 = dh1 * dsilu(z1)
    g[OFF["b1"][0]:OFF["b1"][1]] = d1.sum(axis=0)
    d1b = bf16(d1)
    g[OFF["W1"][0]:OFF["W1"][1]] = (d1b.T @ x).ravel()
    return g, float((e * e).sum())
