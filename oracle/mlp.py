"""CPU oracle of the closure network -- test infrastructure, never the
product path.

The network is the one the device trains and evaluates: n_in -> width ->
width -> width -> n_out, GELU in its tanh form after each hidden layer,
linear output; the loss is the mean squared error over the first ``nreal``
outputs, L = sum_(n, j<nreal) (y - t)^2 / (N nreal).  Here everything is
FP64 without any rounding to BF16: the exact arithmetic the device's BF16
products and FP32 accumulations approximate.  The gradients are the
textbook backward pass of that function; ``fd_grad`` is its central
finite difference, which pins the backward pass (tests/test_oracle_mlp.py).
"""
import math

import numpy as np

C_GELU = math.sqrt(2.0 / math.pi)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def dgelu(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * z * z)


def forward(W, B, x):
    """Pre-activations Z[l] and layer inputs H[l]; W[l] is (in, out)."""
    h, Z, H = np.asarray(x, dtype=np.float64), [], []
    for l in range(len(W)):
        H.append(h)
        z = h @ W[l] + B[l]
        Z.append(z)
        h = gelu(z) if l < len(W) - 1 else z
    return Z, H


def loss(W, B, x, t, nreal):
    y = forward(W, B, x)[0][-1]
    d = y[:, :nreal] - t[:, :nreal]
    return float((d ** 2).sum() / (x.shape[0] * nreal))


def loss_and_grads(W, B, x, t, nreal):
    """(loss, [(dL/dW[l], dL/dB[l]) for each layer])."""
    Z, H = forward(W, B, x)
    n = x.shape[0]
    y = Z[-1]
    d = np.zeros_like(y)
    d[:, :nreal] = y[:, :nreal] - t[:, :nreal]
    dz = 2.0 * d / (n * nreal)
    grads = [None] * len(W)
    for l in range(len(W) - 1, -1, -1):
        grads[l] = (H[l].T @ dz, dz.sum(axis=0))
        if l > 0:
            dz = (dz @ W[l].T) * dgelu(Z[l - 1])
    return float((d ** 2).sum() / (n * nreal)), grads


def fd_grad(W, B, x, t, nreal, layer, index, is_bias=False, h=1e-6):
    """Central difference of the loss in one weight (index a (i, j) pair) or
    bias (index j) of ``layer``."""
    W = [w.copy() for w in W]
    B = [b.copy() for b in B]
    P = B[layer] if is_bias else W[layer]
    v = P[index]
    P[index] = v + h
    lp = loss(W, B, x, t, nreal)
    P[index] = v - h
    lm = loss(W, B, x, t, nreal)
    P[index] = v
    return (lp - lm) / (2.0 * h)
