"""CPU oracle for the closure network (TEST INFRASTRUCTURE ONLY: used by tests/
and bench.py's checks, never by the product).

A float64 numpy restatement of the MLP of include/ce_closure.h: layers
[W_l (fan_out x fan_in), b_l], SiLU on hidden layers, linear output, loss
sum(weight * (out - target)^2). With bf16=True the activations are rounded to
bfloat16 at the same points the GPU kernels round them (weights, Z, H, and the
back-propagated pre-activation gradients), so gradients can be compared tightly.
"""
from __future__ import annotations

import numpy as np


def to_bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def unpack(params: np.ndarray, in_dim: int, hidden: int, depth: int, out_dim: int):
    dims = [in_dim] + [hidden] * depth + [out_dim]
    ws, bs, o = [], [], 0
    for l in range(depth + 1):
        fi, fo = dims[l], dims[l + 1]
        ws.append(params[o:o + fi * fo].reshape(fo, fi).astype(np.float64))
        o += fi * fo
        bs.append(params[o:o + fo].astype(np.float64))
        o += fo
    return ws, bs


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, in_dim, hidden, depth, out_dim, bf16=False):
    ws, bs = unpack(params, in_dim, hidden, depth, out_dim)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    h = r(x)
    zs, hs = [], [h]
    for l in range(depth):
        z = r(h @ r(ws[l]).T + bs[l])
        h = r(silu(z))
        zs.append(z)
        hs.append(h)
    out = h @ r(ws[depth]).T + bs[depth]
    return out, zs, hs


def gradients(params, x, target, weight, in_dim, hidden, depth, out_dim, bf16=False):
    """(loss, flat gradient in parameter layout)."""
    ws, _ = unpack(params, in_dim, hidden, depth, out_dim)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    out, zs, hs = forward(params, x, in_dim, hidden, depth, out_dim, bf16)
    d = out - target
    loss = float(np.sum(weight * d * d))
    dcur = r(2.0 * weight * d)
    gws, gbs = [None] * (depth + 1), [None] * (depth + 1)
    for l in range(depth, -1, -1):
        gws[l] = dcur.T @ hs[l]
        gbs[l] = dcur.sum(axis=0)
        if l == 0:
            break
        dcur = r((dcur @ r(ws[l])) * dsilu(zs[l - 1]))
    flat = np.concatenate([np.concatenate([gws[l].ravel(), gbs[l]]) for l in range(depth + 1)])
    return loss, flat
