"""CPU restatement of the learned guide's network for the GPU checks.

The same computation as spatial_query_b200/csrc/guide.cu in float64 (numpy),
with the GPU's rounding points kept: features in float32, weights and every
activation that feeds a GEMM rounded to bf16 (round to nearest even), the
pre-activation bias added in float32, dZ of each layer rounded to bf16 before
it feeds the weight and input gradients. Parameter vectors use the C ABI's
host layout: W1 [128 x 6], b1, W2 [128 x 128], b2, W3, b3, W4 [n_out x 128], b4.
"""
from __future__ import annotations

import numpy as np

H = 128
IN = 6


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bf16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray, n_out: int) -> dict:
    o = 0
    out = {}
    for name, shape in (("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
                        ("W4", (n_out, H)), ("b4", (n_out,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape).astype(np.float32)
        o += n
    assert o == p.size
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")]).astype(np.float32)


def features(rays: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """Origin to [-1, 1] over the scene box, direction as is (float32 steps)."""
    rays = rays.astype(np.float32)
    lo = lo.astype(np.float32)
    ext = (hi.astype(np.float32) - lo)
    inv = np.where(ext > 0, np.float32(1.0) / np.where(ext > 0, ext, np.float32(1.0)), np.float32(0.0)).astype(np.float32)
    o = ((rays[:, :3] - lo) * inv).astype(np.float32)
    o = (o * np.float32(2.0)).astype(np.float32) - np.float32(1.0)
    return np.concatenate([o, rays[:, 3:6]], axis=1).astype(np.float32)


def forward(p: dict, x: np.ndarray):
    """Activations (bf16-rounded) and the float64 logits."""
    a = bf16(x).astype(np.float64)
    acts = [a]
    for l in (1, 2, 3):
        z = (a @ bf16(p[f"W{l}"]).astype(np.float64).T).astype(np.float32) + p[f"b{l}"]
        a = bf16(np.maximum(z, 0.0)).astype(np.float64)
        acts.append(a)
    logits = a @ bf16(p["W4"]).astype(np.float64).T + p["b4"].astype(np.float64)
    return acts, logits


def loss_and_grads(p: dict, x: np.ndarray, labels: np.ndarray, n_buckets: int):
    acts, logits = forward(p, x)
    B, n_out = logits.shape
    valid = (labels >= 0) & (labels < n_buckets)
    n_lab = max(int(valid.sum()), 1)
    lg = logits[:, :n_buckets]
    m = lg.max(axis=1, keepdims=True)
    e = np.exp(lg - m)
    s = e.sum(axis=1, keepdims=True)
    prob = e / s
    y = np.where(valid, labels, 0)
    loss = float(((np.log(s[:, 0]) + m[:, 0] - lg[np.arange(B), y]) * valid).sum() / n_lab)
    d = np.zeros((B, n_out))
    d[:, :n_buckets] = prob
    d[np.arange(B), y] -= 1.0
    d[~valid] = 0.0
    dz = bf16((d / n_lab).astype(np.float32)).astype(np.float64)
    g = {"b4": dz.sum(axis=0), "W4": dz.T @ acts[3]}
    dh = dz @ bf16(p["W4"]).astype(np.float64)
    for l in (3, 2, 1):
        dz = bf16(np.where(acts[l] > 0, dh, 0.0).astype(np.float32)).astype(np.float64)
        g[f"b{l}"] = dz.sum(axis=0)
        g[f"W{l}"] = dz.T @ acts[l - 1][:, : (IN if l == 1 else H)]
        if l > 1:
            dh = dz @ bf16(p[f"W{l}"]).astype(np.float64)
    return loss, g
