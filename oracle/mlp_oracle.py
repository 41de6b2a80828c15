"""CPU oracle of the learned-kappa MLP training step (test infrastructure only).

numpy restatement of imcom_b200/csrc/kappa.cu's mlp_grad_kernel: the same
bf16 rounding points (inputs, weights, hidden activations; round to nearest
even), ReLU masks taken on the rounded activations, the same loss
(o0 - t)^2 + 0.25 (o1 - log(|o0 - t| + 0.01))^2 with the second target held
fixed, and the gradient with respect to the bf16-rounded weights.
Arithmetic in float64, so the GPU's fp32 sums agree to ~1e-6.
"""
from __future__ import annotations

import numpy as np

NF, NH, NO = 12, 64, 2


def bf16(x):
    a = np.asarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    o, out = 0, []
    for shape in ((NH, NF), (NH,), (NH, NH), (NH,), (NO, NH), (NO,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def loss_and_grad(params, feat, target, round_bf16=True, frozen_lt=None):
    """feat (12, N) normalised features, target (N).  Returns (summed loss,
    packed gradient).  round_bf16=False drops every rounding (for finite-
    difference checks of the backward algebra); frozen_lt fixes the second
    head's target (the kernel treats it as a constant)."""
    rnd = bf16 if round_bf16 else (lambda x: np.asarray(x, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(params)
    W1r, W2r, W3r = rnd(W1), rnd(W2), rnd(W3)
    b1d, b2d, b3d = (np.asarray(b, dtype=np.float64) for b in (b1, b2, b3))
    X = rnd(feat).T                                    # (N, 12)
    H1 = rnd(np.maximum(X @ W1r.T + b1d, 0.0))         # (N, 64)
    H2 = rnd(np.maximum(H1 @ W2r.T + b2d, 0.0))
    O = H2 @ W3r.T + b3d                               # (N, 2)
    e = O[:, 0] - np.asarray(target, dtype=np.float64)
    lt = np.log(np.abs(e) + 0.01) if frozen_lt is None else frozen_lt
    e1 = O[:, 1] - lt
    loss = float(np.sum(e * e + 0.25 * e1 * e1))
    dO = np.stack([2.0 * e, 0.5 * e1], axis=1)
    gW3 = dO.T @ H2
    gb3 = dO.sum(axis=0)
    D2 = (dO @ W3r) * (H2 > 0)
    gW2 = D2.T @ H1
    gb2 = D2.sum(axis=0)
    D1 = (D2 @ W2r) * (H1 > 0)
    gW1 = D1.T @ X
    gb1 = D1.sum(axis=0)
    g = np.concatenate([x.ravel() for x in (gW1, gb1, gW2, gb2, gW3, gb3)])
    loss_and_grad.last_lt = lt
    return loss, g


def forward(params, feat):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    X = bf16(feat).T
    H1 = bf16(np.maximum(X @ bf16(W1).T + b1, 0.0))
    H2 = bf16(np.maximum(H1 @ bf16(W2).T + b2, 0.0))
    return H2 @ bf16(W3).T + b3
