"""CPU oracle of the boundary MLP (test infrastructure only: the tests import
it as the checker of the library's MLP kernels; nothing in the product
imports it).

FP64 numpy restatement of the network the library trains and applies
(include/nexd.h, learned absorbing boundary): n_in -> H -> H -> n_in, GELU
(0.5 z (1 + erf(z / sqrt 2))), parameters [W1 (H x n_in), b1, W2 (H x H), b2,
W3 (n_in x H), b3] row-major, loss = mean over the batch of |y - t|^2.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf)


def unpack(p, nin, h):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((h, nin), (h,), (h, h), (h,), (nin, h), (nin,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size
    return out


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, x, nin, h):
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, h)
    z1 = x @ W1.T + b1
    a1 = gelu(z1)
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    return a2 @ W3.T + b3, (z1, a1, z2, a2)


def loss_grad(p, x, t, nin, h):
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, h)
    y, (z1, a1, z2, a2) = forward(p, x, nin, h)
    B = x.shape[0]
    loss = ((y - t) ** 2).sum() / B
    dy = 2.0 * (y - t) / B
    gW3, gb3 = dy.T @ a2, dy.sum(axis=0)
    d2 = (dy @ W3) * gelu_grad(z2)
    gW2, gb2 = d2.T @ a1, d2.sum(axis=0)
    d1 = (d2 @ W2) * gelu_grad(z1)
    gW1, gb1 = d1.T @ x, d1.sum(axis=0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g
