"""CPU restatement (numpy, float64) of the CALPHAD surrogate network and of
its gradient, the checker of the library's rs_mlp_grad / rs_mlp_forward
kernels (test infrastructure only).

Layout of the flat parameter vector: W1[32][3], b1[32], W2[32][32], b2[32],
W3[2][32], b3[2]; loss = sum over samples of |out - (y - y_mean) / y_scale|^2.
"""
import numpy as np

H = 32


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + H * 3].reshape(H, 3); o += H * 3
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    W3 = w[o:o + 2 * H].reshape(2, H); o += 2 * H
    b3 = w[o:o + 2]
    return W1, b1, W2, b2, W3, b3


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z1 = x @ W1.T + b1
    a1 = silu(z1)
    z2 = a1 @ W2.T + b2
    a2 = silu(z2)
    return a2 @ W3.T + b3, (z1, a1, z2, a2)


def loss_and_grad(w, x, y, y_mean, y_scale):
    x = np.asarray(x, dtype=np.float64)
    yt = (np.asarray(y, dtype=np.float64) - np.asarray(y_mean)) / np.asarray(y_scale)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    o, (z1, a1, z2, a2) = forward(w, x)
    e = o - yt
    g3 = 2.0 * e
    g2 = (g3 @ W3) * silu_grad(z2)
    g1 = (g2 @ W2) * silu_grad(z1)
    grads = [g1.T @ x, g1.sum(0), g2.T @ a1, g2.sum(0), g3.T @ a2, g3.sum(0)]
    return float((e ** 2).sum()), np.concatenate([g.ravel() for g in grads])
