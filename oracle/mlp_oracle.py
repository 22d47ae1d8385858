"""ORACLE - test infrastructure.  Numpy restatement of the learned closure's network
(retainwall_code_b200 rw_mlp_*): its forward pass and the gradient of its mean squared
error, in two forms:

- ``emulate=True`` repeats the device arithmetic: BF16 (round to nearest even) weights,
  inputs, hidden activations and backward signals, FP32 products and sums, the SiLU
  written as z (1/2 + tanh(z/2) / 2);
- ``emulate=False`` is plain float64, the reference for finite-difference checks.

Used only by tests/ as the checker of the tensor-core kernels."""
from __future__ import annotations

import numpy as np

IN, HID, OUT, NHID = 16, 64, 6, 4
P_W1 = 0
P_B1 = P_W1 + IN * HID
P_W2 = P_B1 + HID
P_B2 = P_W2 + HID * HID
P_W3 = P_B2 + HID
P_B3 = P_W3 + HID * HID
P_W4 = P_B3 + HID
P_B4 = P_W4 + HID * HID
P_W5 = P_B4 + HID
P_B5 = P_W5 + HID * OUT
NPARAM = P_B5 + OUT
SHAPES = [(P_W1, (IN, HID)), (P_B1, (HID,)), (P_W2, (HID, HID)), (P_B2, (HID,)), (P_W3, (HID, HID)), (P_B3, (HID,)),
          (P_W4, (HID, HID)), (P_B4, (HID,)), (P_W5, (HID, OUT)), (P_B5, (OUT,))]


def bf16(a) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p)
    out = []
    for off, shp in SHAPES:
        n = int(np.prod(shp))
        out.append(p[off:off + n].reshape(shp))
    Ws = out[0::2]
    bs = out[1::2]
    return Ws, bs


def pack(Ws, bs) -> np.ndarray:
    p = np.zeros(NPARAM, np.float64)
    for (off, shp), a in zip(SHAPES, [x for pair in zip(Ws, bs) for x in pair]):
        p[off:off + int(np.prod(shp))] = np.asarray(a).ravel()
    return p


def _sig(z):
    return 0.5 + 0.5 * np.tanh(0.5 * z)


def forward(p, X, emulate=True):
    """Outputs (n, 6) and the cache of the backward pass."""
    Ws, bs = unpack(p)
    if emulate:
        f = np.float32
        Ws = [bf16(W) for W in Ws]
        bs = [np.asarray(b, f) for b in bs]
        H = bf16(X)
    else:
        f = np.float64
        Ws = [np.asarray(W, f) for W in Ws]
        bs = [np.asarray(b, f) for b in bs]
        H = np.asarray(X, f)
    hs, zs = [H], []
    for l in range(NHID):
        Z = (H.astype(f) @ Ws[l].astype(f)).astype(f) + bs[l]
        A = Z * _sig(Z)
        H = bf16(A) if emulate else A
        zs.append(Z)
        hs.append(H)
    Y = (H @ Ws[NHID]).astype(f) + bs[NHID]
    return Y, (Ws, bs, hs, zs, f)


def loss_grad(p, X, T, emulate=True):
    """Mean squared error over samples and outputs, and its gradient (NPARAM)."""
    Y, (Ws, bs, hs, zs, f) = forward(p, X, emulate)
    n = len(X)
    D = Y - np.asarray(T, f)
    loss = float(np.mean(D.astype(np.float64) ** 2))
    G = (2.0 * D / (n * OUT)).astype(f)
    if emulate:
        G = bf16(G)
    dWs, dbs = [None] * (NHID + 1), [None] * (NHID + 1)
    dWs[NHID] = hs[NHID].T @ G
    dbs[NHID] = G.sum(0)
    dH = G @ Ws[NHID].T
    for l in range(NHID - 1, -1, -1):
        Z = zs[l]
        s = _sig(Z)
        G = (dH * (s + Z * s * (1.0 - s))).astype(f)
        if emulate:
            G = bf16(G)
        dWs[l] = hs[l].T @ G
        dbs[l] = G.sum(0)
        if l > 0:
            dH = G @ Ws[l].T
    return loss, pack(dWs, dbs)
