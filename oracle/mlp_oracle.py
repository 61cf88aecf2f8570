"""CPU oracle of the twist-surrogate MLP (test infrastructure only).

Float64 numpy restatement of the network, loss and optimiser that the
library's ftlm_mlp_* calls run on the GPU: x[n_in] -> `depth` tanh layers of
`width` -> linear y[n_out]; parameters are one flat vector, per layer W[out][in]
then b[out]; loss sum(mask * (y - t)^2) / sum(mask); Adam with
b1 = 0.9, b2 = 0.999, eps = 1e-8 and bias correction. The surrogate has no
counterpart in the reference, so this oracle is pinned by finite differences
of its own loss (tests/test_mlp_oracle.py), not by reference vectors.
"""
from __future__ import annotations

import numpy as np


def layer_shapes(n_in, width, depth, n_out):
    fi = [n_in] + [width] * depth
    fo = [width] * depth + [n_out]
    return list(zip(fi, fo))


def num_params(n_in, width, depth, n_out):
    return sum(i * o + o for i, o in layer_shapes(n_in, width, depth, n_out))


def unpack(p, shapes):
    out, off = [], 0
    for i, o in shapes:
        W = p[off:off + i * o].reshape(o, i)
        off += i * o
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def forward(p, shapes, x):
    """Activations of every layer (the last one is the output)."""
    acts = []
    h = np.asarray(x, np.float64)
    layers = unpack(np.asarray(p, np.float64), shapes)
    for l, (W, b) in enumerate(layers):
        z = h @ W.T + b
        h = np.tanh(z) if l + 1 < len(layers) else z
        acts.append(h)
    return acts


def loss_grad(p, shapes, x, t, mask):
    """(loss, flat gradient) of the masked mean squared error."""
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    m = np.asarray(mask, np.float64)
    acts = forward(p, shapes, x)
    layers = unpack(np.asarray(p, np.float64), shapes)
    cnt = m.sum()
    y = acts[-1]
    loss = float((m * (y - t) ** 2).sum() / cnt)
    dz = 2.0 * m * (y - t) / cnt
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        hin = x if l == 0 else acts[l - 1]
        grads[l] = (dz.T @ hin, dz.sum(0))
        if l > 0:
            dz = (dz @ W) * (1.0 - acts[l - 1] ** 2)
    g = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, g


def adam_steps(p, shapes, batches, lr, b1=0.9, b2=0.999, eps=1e-8):
    """Adam over a sequence of (x, t, mask) batches from zero moments."""
    p = np.array(p, np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for step, (x, t, mask) in enumerate(batches, start=1):
        _, g = loss_grad(p, shapes, x, t, mask)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        p -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p
