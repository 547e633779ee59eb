"""Float64 numpy restatement of the surrogate network's forward and backward passes (test
infrastructure: the CPU reference the tensor-core kernels' outputs and gradients are checked
against). Same architecture: x -> [W x + b -> SiLU] x 4 -> W x + b, mean-squared-error loss."""
import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, X):
    """params: [(W [out, in], b [out])] per layer. Returns (y, cache)."""
    h = X
    zs, hs = [], [X]
    for W, b in params[:-1]:
        z = h @ W.T + b
        zs.append(z)
        h = silu(z)
        hs.append(h)
    W, b = params[-1]
    return h @ W.T + b, (zs, hs)


def loss_and_grads(params, X, T):
    """Mean over samples and outputs of the squared error, and its gradients per layer."""
    y, (zs, hs) = forward(params, X)
    n, m = T.shape
    loss = float(np.mean((y - T) ** 2))
    d = 2.0 * (y - T) / (n * m)
    grads = [None] * len(params)
    for l in range(len(params) - 1, -1, -1):
        W, _ = params[l]
        grads[l] = (d.T @ hs[l], d.sum(0))
        if l > 0:
            d = (d @ W) * silu_grad(zs[l - 1])
    return loss, grads
