"""CPU oracle of the learned-guess network (test infrastructure only).

Restates, in numpy float64, the forward pass, the mean-squared-error
gradients and the Adam step that csrc/pfk_mlp.cu runs on the tensor cores.
It rounds to bfloat16 (round to nearest even) at the same points as the
device: the network input, the weights used in the products, the hidden
activations and the output-side gradient that enters each product.  All
other arithmetic is float64, so device-oracle differences measure the
device's FP32 accumulation only.  The reference has no network (the learned
guess is an addition behind its ReadDensity guess path, scf.cpp:213-216), so
this oracle is pinned by a finite-difference check of its own gradients in
tests/test_mlp_oracle.py.
"""
import numpy as np


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    x = np.asarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(dims, p):
    out, o = [], 0
    for din, dout in zip(dims[:-1], dims[1:]):
        W = np.asarray(p[o:o + din * dout], dtype=np.float64).reshape(din, dout)
        o += din * dout
        b = np.asarray(p[o:o + dout], dtype=np.float64)
        o += dout
        out.append((W, b))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(dims, p, X, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(dims, p)
    H = [r(X)]
    Z = []
    for l, (W, b) in enumerate(layers):
        z = H[-1] @ r(W) + b
        Z.append(z)
        if l < len(layers) - 1:
            H.append(r(silu(z)))
    return Z[-1], Z, H


def gradients(dims, p, X, T, rounding=True):
    """(parameter-vector gradient, loss) of mean((Y - T)^2)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(dims, p)
    Y, Z, H = forward(dims, p, X, rounding)
    n = Y.size
    resid = Y - np.asarray(T, dtype=np.float64)
    loss = float((resid * resid).sum() / n)
    dZ = 2.0 * resid / n
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        G = r(dZ)
        grads[l] = (H[l].T @ G, dZ.sum(axis=0))
        if l == 0:
            break
        dH = G @ r(W).T
        dZ = dH * silu_grad(Z[l - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return flat, loss


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
