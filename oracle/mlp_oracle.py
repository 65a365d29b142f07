"""CPU oracle of the learned potential's network (test infrastructure: only tests/ use it).

The network of include/spo_mlp.h restated in numpy float64, with the device's rounding points: inputs,
weights and the hidden activations are rounded to BF16 (round to nearest even) where the device
stores them as BF16, everything else is exact. Parameters are in spo_mlp_get_parameters' order:
layer by layer W (out x in, the first layer's in = the padded input width) then b, then the output
weights w_out (width) and b_out.

There is no reference counterpart: the reference evaluates its potential exactly
(src/potential/potential_grid.hpp:48-55). ``gradients`` is checked against finite differences
(tests/test_mlp_oracle.py); the device's gradients are checked against it.
"""

from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray, n_pad: int, width: int, depth: int):
    layers, off = [], 0
    for l in range(depth):
        k = n_pad if l == 0 else width
        w = p[off:off + width * k].reshape(width, k).astype(np.float64)
        off += width * k
        b = p[off:off + width].astype(np.float64)
        off += width
        layers.append((w, b))
    wo = p[off:off + width].astype(np.float64)
    bo = float(p[off + width])
    assert off + width + 1 == p.size
    return layers, wo, bo


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, n_pad, width, depth, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers, wo, bo = unpack(p, n_pad, width, depth)
    a = np.zeros((x.shape[0], n_pad))
    a[:, :x.shape[1]] = x
    a = r(a)
    zs, acts = [], [a]
    for w, b in layers:
        z = a @ r(w).T + b
        a = r(silu(z))
        zs.append(z)
        acts.append(a)
    out = a @ wo + bo
    return out, zs, acts


def gradients(p, x, y, n_pad, width, depth, rounding=True):
    """Loss (mean squared error) and its gradient, in parameter order."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    layers, wo, bo = unpack(p, n_pad, width, depth)
    out, zs, acts = forward(p, x, n_pad, width, depth, rounding)
    n = x.shape[0]
    e = out - y
    loss = float(np.mean(e * e))
    d = 2.0 * e / n
    g_wo = acts[-1].T @ d
    g_bo = d.sum()
    g = d[:, None] * wo[None, :]
    grads = [None] * depth
    for l in range(depth - 1, -1, -1):
        w, _ = layers[l]
        dz = g * silu_grad(zs[l])
        gb = dz.sum(axis=0)
        dz16 = r(dz)
        gw = dz16.T @ acts[l]
        grads[l] = (gw, gb)
        if l > 0:
            g = r(dz16 @ r(w))
    flat = []
    for gw, gb in grads:
        flat += [gw.ravel(), gb]
    flat += [g_wo, np.array([g_bo])]
    return loss, np.concatenate(flat)
