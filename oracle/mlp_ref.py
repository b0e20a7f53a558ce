"""CPU restatement of one training step of the learned correction's MLP —
TEST INFRASTRUCTURE ONLY (the gradient check of the GPU training kernels).

The network, its parameter layout and the BF16 / quantization-aware forward
follow the library's training module: W1[32][16] (columns 14, 15 zero),
b1[32], W2[32][32], b2[32], W3[8][32] (row 7 zero), b3[8]; inputs
u = clamp(x / s_in, +-127) / 127 (BF16-rounded, or on the int8 grid under
QAT), hidden units relu with BF16-rounded (or int8-grid) activations, output
y = W3 h2 + b3, loss = mean Huber(y - t / s_t) over samples x 7 blocks. The
forward sums are FP32 fused multiply-adds in the kernel's order, emulated
here in float64 with one rounding to float32 per step. The reference project
has no learned predictor; this is the oracle of this library's own part.
"""
from __future__ import annotations

import numpy as np

PW1, PB1, PW2, PB2, PW3, PB3, NP = 0, 512, 544, 1568, 1600, 1856, 1864


def bf16(a):
    """Round float32 values to BF16 (nearest even), returned as float32."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32)
    return np.where(np.isfinite(a), out, a).astype(np.float32)


def _fma_chain(acc, w, x):
    """acc + sum_k w[k] * x[:, k] as successive float32 FMAs."""
    acc = acc.astype(np.float32)
    for k in range(w.shape[0]):
        acc = (w[k].astype(np.float64) * x[:, k].astype(np.float64) + acc.astype(np.float64)).astype(np.float32)
    return acc


def forward_weights(params, qat):
    p = np.asarray(params, np.float32).copy()
    tensors = [(PW1, PB1), (PW2, PB2), (PW3, PB3)]
    for b, e in tensors:
        w = p[b:e]
        if qat:
            step = np.float32(np.float32(np.abs(w).max()) / np.float32(127.0))
            p[b:e] = np.rint(w / step).astype(np.float32) * step if step > 0 else 0.0
        else:
            p[b:e] = bf16(w)
    return p


def step(params, x, t, s_in, s_t, delta, qat=False, sa=(1.0, 1.0)):
    """Mean loss and dL/dparams (float64) of one batch; x (n, 16) features in
    eb (BF16-rounded first, as the kernel stores them), t (n, 8)."""
    Wf = forward_weights(params, qat)
    W1 = Wf[PW1:PB1].reshape(32, 16)
    b1 = Wf[PB1:PW2]
    W2 = Wf[PW2:PB2].reshape(32, 32)
    b2 = Wf[PB2:PW3]
    W3 = Wf[PW3:PB3].reshape(8, 32)
    b3 = Wf[PB3:NP]
    n = x.shape[0]
    xs = bf16(np.asarray(x, np.float32))
    inv_s_in, inv_s_t = np.float32(1.0 / s_in), np.float32(1.0 / s_t)
    dlt = np.float32(delta / s_t)
    q = xs[:, :14] * inv_s_in
    if qat:
        q = np.rint(q)
    q = np.clip(q, -127, 127).astype(np.float32)
    u = q * np.float32(1.0 / 127.0)
    if not qat:
        u = bf16(u)
    u = np.concatenate([u, np.zeros((n, 2), np.float32)], axis=1)

    def act(pre, s):
        if qat:
            s = np.float32(s)
            return (np.clip(np.rint(pre / s), 0, 127).astype(np.float32) * s, (pre > 0) & (pre < np.float32(127.0) * s))
        return np.where(pre > 0, bf16(pre), 0).astype(np.float32), pre > 0

    pre1 = np.stack([_fma_chain(np.full(n, b1[j], np.float32), W1[j, :14], u[:, :14]) for j in range(32)], axis=1)
    h1, m1 = act(pre1, sa[0])
    pre2 = np.stack([_fma_chain(np.full(n, b2[j], np.float32), W2[j], h1) for j in range(32)], axis=1)
    h2, m2 = act(pre2, sa[1])
    y = np.stack([_fma_chain(np.full(n, b3[b], np.float32), W3[b], h2) for b in range(7)], axis=1)
    e = (y - np.asarray(t, np.float32)[:, :7] * inv_s_t).astype(np.float64)
    ae = np.abs(e)
    loss = np.where(ae <= dlt, 0.5 * e * e, dlt * (ae - 0.5 * dlt)).sum() / (n * 7)
    dy = np.clip(e, -dlt, dlt) / (n * 7)
    dh2 = (dy @ W3[:7].astype(np.float64)) * m2
    dh1 = (dh2 @ W2.astype(np.float64)) * m1
    g = np.zeros(NP)
    gw1 = dh1.T @ u.astype(np.float64)
    gw1[:, 14:] = 0
    g[PW1:PB1] = gw1.ravel()
    g[PB1:PW2] = dh1.sum(0)
    g[PW2:PB2] = (dh2.T @ h1.astype(np.float64)).ravel()
    g[PB2:PW3] = dh2.sum(0)
    gw3 = np.zeros((8, 32))
    gw3[:7] = dy.T @ h2.astype(np.float64)
    g[PW3:PB3] = gw3.ravel()
    g[PB3:PB3 + 7] = dy.sum(0)
    return loss, g
