"""TEST INFRASTRUCTURE ONLY -- FP64 CPU oracle of the user encoder's loss and
gradients, used to check the GPU's forward/backward kernels.

The encoder has no counterpart in the reference. Its definition:
  h0 = mean over the user's training ratings of E_item[5 i + r - 1] + E_rate[r-1] + E_date[b]
  (E_item has one row per (item, rating) pair)
  z1 = h0 W1 + b1, h1 = GELU(z1); z2 = h1 W2 + b2, h2 = GELU(z2); y = h2 W3 + b3
  loss = mean((y - t)^2) over the batch and the f+2 outputs, t standardised.
With mimic_bf16 the oracle rounds to BF16 exactly where the GPU stores BF16
(GEMM operands: weights, h0, h1, h2, dy, dz1, dz2), so the remaining
difference is FP32 versus FP64 accumulation; without it, it is the plain FP64
model and the difference also contains the BF16 rounding itself.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def loss_and_grads(params, hist, targets, mimic_bf16=True):
    """params: dict of FP32 arrays (e_item, e_rate, e_date, w1, b1, w2, b2, w3, b3);
    hist: list of (items, ratings 1..5, time bins) per user; targets: [n, O]
    standardised. Returns (loss, grads dict)."""
    r = bf16 if mimic_bf16 else (lambda v: np.asarray(v, np.float64))
    P = {k: np.asarray(v, np.float64) for k, v in params.items()}
    n = len(hist)
    h0 = np.zeros((n, 128))
    for k, (it, rt, tb) in enumerate(hist):
        if len(it):
            h0[k] = (P["e_item"][5 * it + rt - 1] + P["e_rate"][rt - 1] + P["e_date"][tb]).sum(0) / len(it)
    if mimic_bf16:  # the GPU accumulates h0 in FP32 and stores that value
        h0 = h0.astype(np.float32).astype(np.float64)
    W1, W2, W3 = r(P["w1"]), r(P["w2"]), r(P["w3"])
    h0b = r(h0)
    z1 = h0b @ W1 + P["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W2 + P["b2"]
    h2 = r(gelu(z2))
    y = h2 @ W3 + P["b3"]
    t = np.asarray(targets, np.float64)
    O = y.shape[1]
    d = y - t
    loss = float((d * d).sum() / (n * O))
    dy = 2.0 * d / (n * O)
    dyb = r(dy)
    g = {}
    g["w3"] = h2.T @ dyb
    g["b3"] = dy.sum(0)
    dh2 = dyb @ W3.T
    dz2 = r(dh2 * gelu_grad(z2))
    g["w2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dh1 = dz2 @ W2.T
    dz1 = r(dh1 * gelu_grad(z1))
    g["w1"] = h0b.T @ dz1
    g["b1"] = dz1.sum(0)
    dh0 = dz1 @ W1.T
    ge_item = np.zeros_like(P["e_item"])
    ge_rate = np.zeros_like(P["e_rate"])
    ge_date = np.zeros_like(P["e_date"])
    for k, (it, rt, tb) in enumerate(hist):
        if not len(it):
            continue
        dk = dh0[k] / len(it)
        np.add.at(ge_item, 5 * it + rt - 1, dk)
        np.add.at(ge_rate, rt - 1, dk)
        np.add.at(ge_date, tb, dk)
    g["e_item"], g["e_rate"], g["e_date"] = ge_item, ge_rate, ge_date
    return loss, g
