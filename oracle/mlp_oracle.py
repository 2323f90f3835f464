"""CPU oracle for the warm-start network — test infrastructure only.

The reference has no learned component (its GMRES starts from a zero guess,
2S/main.cpp:1067-1075), so this oracle restates the network's mathematical
definition in FP64 numpy: 12 -> 64 -> 64 -> 64 -> 3, SiLU hidden activations,
inputs normalized by (x - mean) / std, loss = mean over batch and components of
(y - t / out_scale)^2, Adam with bias correction (Kingma & Ba 2015, beta1 0.9,
beta2 0.999, eps 1e-8). Parameter layout: W1[12][64] b1[64] W2[64][64] b2[64]
W3[64][64] b3[64] W4[64][3] b4[3], W[i][j] from input i to output j.

It is pinned by a finite-difference check of its own gradient (tests), and
it is the oracle for the CUDA forward, gradient and Adam kernels. Nothing in
the product imports it.
"""
import numpy as np

SHAPES = [(12, 64), (64,), (64, 64), (64,), (64, 64), (64,), (64, 3), (3,)]
NPARAMS = sum(int(np.prod(s)) for s in SHAPES)


def unpack(p):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n], np.float64).reshape(s))
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(a, np.float64).ravel() for a in parts])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, X, mean, std):
    """Returns (y, cache) for inputs X (n x 12)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    x = (np.asarray(X, np.float64) - mean) / std
    z1 = x @ W1 + b1
    a1 = z1 * _sig(z1)
    z2 = a1 @ W2 + b2
    a2 = z2 * _sig(z2)
    z3 = a2 @ W3 + b3
    a3 = z3 * _sig(z3)
    y = a3 @ W4 + b4
    return y, (x, z1, a1, z2, a2, z3, a3)


def _dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(p, X, T, mean, std, out_scale):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    y, (x, z1, a1, z2, a2, z3, a3) = forward(p, X, mean, std)
    e = y - np.asarray(T, np.float64) / out_scale
    n = e.size
    loss = float((e * e).sum() / n)
    d4 = 2.0 * e / n
    d3 = (d4 @ W4.T) * _dsilu(z3)
    d2 = (d3 @ W3.T) * _dsilu(z2)
    d1 = (d2 @ W2.T) * _dsilu(z1)
    g = [x.T @ d1, d1.sum(0), a1.T @ d2, d2.sum(0), a2.T @ d3, d3.sum(0), a3.T @ d4, d4.sum(0)]
    return loss, pack(g)


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step; step counts from 1. Returns (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
