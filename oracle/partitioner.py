"""CPU restatement of the learned-partition kNN's network arithmetic (test
infrastructure only: imported by tests/ as the checker of the device kernels, never by
the product).

kyto has no learned partitioner: this restates the method the device implements, so
its kernels can be checked number for number. Parity here is against this file's own
definition, not against kyto (no kyto code or golden exists for it).

The network: din -> hidden -> hidden -> P, ReLU between, BF16 operands with f32 master
weights. Every operand a device GEMM reads in bf16 is rounded the same way here (round
to nearest, ties to even, on the f32 bits); the sums run in f64 here and in f32 on the
device, so the two agree to f32 accumulation error.
"""

from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round f32 values to bfloat16 (nearest, ties to even), returned as f32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounding = 0x7FFF + ((u >> 16) & 1)
    r = ((u + rounding) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).copy()
    nan = np.isnan(a)
    out[nan] = a[nan]
    return out


class Params:
    """f32 master weights w[l] (out x in) and biases b[l]."""

    def __init__(self, ws: list[np.ndarray], bs: list[np.ndarray]):
        self.w = [np.asarray(w, dtype=np.float32) for w in ws]
        self.b = [np.asarray(b, dtype=np.float32) for b in bs]


def init_params(sizes: list[int], seed: int) -> Params:
    """He-uniform weights, zero biases (tests copy weights to the device, so the two
    generators need not agree)."""
    rng = np.random.default_rng(seed)
    ws, bs = [], []
    for fan_in, fan_out in zip(sizes[:-1], sizes[1:]):
        lim = np.sqrt(6.0 / fan_in)
        ws.append(rng.uniform(-lim, lim, (fan_out, fan_in)).astype(np.float32))
        bs.append(np.zeros(fan_out, dtype=np.float32))
    return Params(ws, bs)


def forward(p: Params, x: np.ndarray):
    """Logits and the cache the backward pass needs: zs[l] (pre-activations, f64 sums of
    bf16 operands) and h[l] (the bf16 inputs of layer l)."""
    h = [bf16(x)]
    zs = []
    n = len(p.w)
    for l in range(n):
        z = h[-1].astype(np.float64) @ bf16(p.w[l]).astype(np.float64).T + p.b[l]
        zs.append(z)
        if l + 1 < n:
            h.append(bf16(np.maximum(z, 0.0).astype(np.float32)))
    return zs[-1], (h, zs)


def softmax(z: np.ndarray) -> np.ndarray:
    m = z.max(axis=1, keepdims=True)
    e = np.exp(z - m)
    return e / e.sum(axis=1, keepdims=True)


def loss_and_grads(p: Params, x: np.ndarray, targets: np.ndarray):
    """Mean soft-target cross-entropy and its gradients with respect to every weight and
    bias: dZ_last = (softmax - T) / B; dW = dZ^T h; db = sum dZ; dh = dZ bf16(W); the
    ReLU passes dZ where z > 0."""
    z, (h, zs) = forward(p, x)
    b = x.shape[0]
    prob = softmax(z)
    loss = float(-(targets * np.log(np.maximum(prob, 1e-30))).sum() / b)
    dz = (prob - targets) / b
    gw = [None] * len(p.w)
    gb = [None] * len(p.w)
    for l in range(len(p.w) - 1, -1, -1):
        gw[l] = dz.T @ h[l].astype(np.float64)
        gb[l] = dz.sum(axis=0)
        if l > 0:
            dh = dz @ bf16(p.w[l]).astype(np.float64)
            dz = dh * (zs[l - 1] > 0.0)
    return loss, gw, gb
