"""ORACLE — test infrastructure only.

FP32 numpy restatement of the learned proposal's scoring network
(glimpse_b200/csrc/mlp.cu): 48 -> 256 -> 256 -> 1 with ReLU, forward, the
weighted binary cross-entropy loss and its gradients. The network has no
counterpart in the reference (which selects states by PBWT alone), so this is
the CPU side of the gradient check, not a reference restatement.

The BF16 rounding points are the GPU's: features, W1 and W2 are rounded to
BF16; layer 1's ReLU output h1 is rounded before layer 2; layer 2's ReLU output
is used in FP32 for the score and rounded to BF16 (h2) for the backward pass;
dL/dz2 and dL/dz1 are rounded to BF16 before the GEMMs that consume them.
Products accumulate in FP32 (float64 here, rounded once).

Packed parameters: W1 [256][64] (columns 48..63 zero), b1 [256], W2 [256][256],
b2 [256], w3 [256], b3 [1].
"""
from __future__ import annotations

import numpy as np

N_IN, N_INP, N_HID = 48, 64, 256
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_HID * N_INP
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID
N_PARAMS = OFF_B3 + 1


def bf16(a):
    """Round float32 values to BF16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p, np.float32)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(N_HID, N_INP), b1=p[OFF_B1:OFF_W2], W2=p[OFF_W2:OFF_B2].reshape(N_HID, N_HID),
                b2=p[OFF_B2:OFF_W3], w3=p[OFF_W3:OFF_B3], b3=p[OFF_B3:])


def pack(W1, b1, W2, b2, w3, b3):
    return np.concatenate([np.asarray(W1, np.float32).ravel(), b1, np.asarray(W2, np.float32).ravel(), b2, w3,
                           np.atleast_1d(np.float32(b3))]).astype(np.float32)


def _mm(a, b):
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward(p, x):
    """Scores and the intermediate values of the GPU's forward pass for rows x (n, 48)."""
    P = unpack(p)
    n = x.shape[0]
    xb = np.zeros((n, N_INP), np.float32)
    xb[:, :N_IN] = bf16(x)
    W1b, W2b = bf16(P["W1"]), bf16(P["W2"])
    h1 = bf16(np.maximum(_mm(xb, W1b.T) + P["b1"], 0.0))
    h2f = np.maximum(_mm(h1, W2b.T) + P["b2"], 0.0)
    score = (h2f.astype(np.float64) @ P["w3"].astype(np.float64)).astype(np.float32) + P["b3"][0]
    return dict(xb=xb, W1b=W1b, W2b=W2b, h1=h1, h2f=h2f, h2=bf16(h2f), score=score)


def loss_and_grad(p, x, y, wt=None):
    """Mean weighted BCE-with-logits loss and the packed FP32 gradient."""
    P = unpack(p)
    f = forward(p, x)
    n = x.shape[0]
    y = np.asarray(y, np.float32)
    wt = np.ones(n, np.float32) if wt is None else np.asarray(wt, np.float32)
    s = f["score"].astype(np.float64)
    loss = float(np.sum(wt * (np.maximum(s, 0) - s * y + np.log1p(np.exp(-np.abs(s))))) / n)
    pr = 1.0 / (1.0 + np.exp(-s))
    ds = ((pr - y) * wt / n).astype(np.float32)
    h2 = f["h2"]
    dz2f = np.where(h2 > 0, ds[:, None] * P["w3"][None, :], 0.0).astype(np.float32)
    dz2 = bf16(dz2f)
    g_w3 = (ds.astype(np.float64) @ h2.astype(np.float64)).astype(np.float32)
    g_b2 = dz2f.astype(np.float64).sum(0).astype(np.float32)
    g_b3 = np.float32(ds.astype(np.float64).sum())
    g_W2 = _mm(dz2.T, f["h1"])
    dh1 = _mm(dz2, f["W2b"])
    dz1 = bf16(np.where(f["h1"] > 0, dh1, 0.0))
    g_b1 = dz1.astype(np.float64).sum(0).astype(np.float32)
    g_W1 = _mm(dz1.T, f["xb"])
    return loss, pack(g_W1, g_b1, g_W2, g_b2, g_w3, g_b3)


def loss_exact(p, x, y, wt=None):
    """The loss in float64 without BF16 rounding (for finite-difference checks of the formulas)."""
    P = {k: v.astype(np.float64) for k, v in unpack(p).items()}
    n = x.shape[0]
    xp = np.zeros((n, N_INP))
    xp[:, :N_IN] = x
    h1 = np.maximum(xp @ P["W1"].T + P["b1"], 0)
    h2 = np.maximum(h1 @ P["W2"].T + P["b2"], 0)
    s = h2 @ P["w3"] + P["b3"][0]
    wt = np.ones(n) if wt is None else np.asarray(wt, np.float64)
    return float(np.sum(wt * (np.maximum(s, 0) - s * y + np.log1p(np.exp(-np.abs(s))))) / n)


def init_params(seed=1):
    """He-uniform weights and zero biases (the same rule as gp_mlp_init, a different generator)."""
    rng = np.random.default_rng(seed)
    W1 = np.zeros((N_HID, N_INP), np.float32)
    W1[:, :N_IN] = rng.uniform(-1, 1, (N_HID, N_IN)) * np.sqrt(6.0 / N_IN)
    W2 = (rng.uniform(-1, 1, (N_HID, N_HID)) * np.sqrt(6.0 / N_HID)).astype(np.float32)
    w3 = (rng.uniform(-1, 1, N_HID) * np.sqrt(3.0 / N_HID)).astype(np.float32)
    return pack(W1, np.zeros(N_HID, np.float32), W2, np.zeros(N_HID, np.float32), w3, 0.0)
