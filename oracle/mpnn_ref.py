"""CPU oracle of the warm-start message-passing network (test infrastructure
only; never imported by the product).  Restates, in float64 numpy, the
network of sdpa_b200/csrc/mpnn.cu with the same parameter layout and the
same BF16 rounding of the weights, forward and backward:

    h_{l+1} = relu(h_l Ws_l^T + (A h_l) Wn_l^T + b_l),  l = 0..2
    r = h_3 w_o + b_o,  loss = sum_i mask_i (r_i - t_i)^2 / count

The network has no counterpart in the reference (the learned warm start is
new); parity of the CUDA kernels is pinned against this restatement and its
own finite-difference gradient check (tests/test_mpnn_oracle.py).
"""
from __future__ import annotations

import numpy as np

H, F0, L = 64, 8, 3


def fin(l):
    return F0 if l == 0 else H


def offsets():
    o, out = 0, []
    for l in range(L):
        ws = o
        wn = ws + H * fin(l)
        b = wn + H * fin(l)
        out.append((ws, wn, b))
        o = b + H
    return out, o, o + H + 1


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even) -> float64."""
    a = np.asarray(w, np.float32).copy()
    u = a.view(np.uint32)
    u += 0x7FFF + ((u >> 16) & 1)
    u &= 0xFFFF0000
    return a.view(np.float32).astype(np.float64)


def unpack(w):
    offs, oo, n = offsets()
    wr = bf16_round(w)
    layers = []
    for l, (ws, wn, b) in enumerate(offs):
        layers.append((wr[ws:wn].reshape(H, fin(l)), wr[wn:b].reshape(H, fin(l)), wr[b:b + H]))
    return layers, wr[oo:oo + H], wr[oo + H]


def adjacency(n, rowptr, col, aval):
    A = np.zeros((n, n))
    for i in range(n):
        for e in range(rowptr[i], rowptr[i + 1]):
            A[i, col[e]] += aval[e]
    return A


def forward(w, feat, A):
    layers, wo, bo = unpack(w)
    hs, aggs, zs = [np.asarray(feat, np.float64)], [], []
    for Ws, Wn, b in layers:
        h = hs[-1]
        agg = A @ h
        z = h @ Ws.T + agg @ Wn.T + b
        aggs.append(agg)
        zs.append(z)
        hs.append(np.maximum(z, 0.0))
    r = hs[-1] @ wo + bo
    return r, (hs, aggs, zs)


def loss_grad(w, feat, A, target, mask):
    """Loss and gradient w.r.t. the (BF16-rounded) parameters, flat layout."""
    layers, wo, bo = unpack(w)
    r, (hs, aggs, zs) = forward(w, feat, A)
    cnt = mask.sum() if mask is not None else len(r)
    m = mask if mask is not None else np.ones_like(r)
    d = (r - target) * m
    loss = float(np.sum(d * d) / cnt)
    dr = 2.0 * d / cnt
    offs, oo, n = offsets()
    g = np.zeros(n)
    g[oo:oo + H] = hs[-1].T @ dr
    g[oo + H] = dr.sum()
    dh = np.outer(dr, wo)
    for l in range(L - 1, -1, -1):
        Ws, Wn, b = layers[l]
        dz = dh * (zs[l] > 0)
        ws, wn, bb = offs[l]
        g[ws:wn] = (dz.T @ hs[l]).ravel()
        g[wn:bb] = (dz.T @ aggs[l]).ravel()
        g[bb:bb + H] = dz.sum(0)
        dh = dz @ Ws + A.T @ (dz @ Wn)
    return loss, g
