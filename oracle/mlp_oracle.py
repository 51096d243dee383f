"""CPU oracle of the warm-start network's forward and backward passes
(TEST INFRASTRUCTURE ONLY).

numpy float64 arithmetic with bf16 rounding applied at exactly the points
where the GPU kernels store bf16 (include/cupf_mlp.h): the pre-activations
z and activations a of the hidden layers and the output-loss gradient.
Everything else (accumulations, bias, the output layer, the weight
gradients) is exact here, so the GPU result differs only by fp32
accumulation order and the rare bf16 rounding flip that causes.

Network: a_0 = x; z_l = a_l W_l^T + b_l; a_{l+1} = gelu(z_l) for the hidden
layers; p = c W_L^T + b_L with c = a_L, or c = [a_L | x] when the output
layer has the input skip; loss = mean over (batch, n_out) of (p - y)^2.
GELU is the erf form 0.5 z (1 + erf(z / sqrt 2)).
"""
from __future__ import annotations

import math

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float64/float32 values to bfloat16 (round to nearest even), back as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> np.uint64(16)) & np.uint64(1)
    r = ((u + np.uint64(0x7FFF) + lsb) >> np.uint64(16)) << np.uint64(16)
    r = np.where(np.isnan(f), u, r)
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward_backward(x, Ws, bs, y, n_out, skip=False):
    """x [B, k0] (bf16 values), Ws[l] [out, in] (bf16 values), bs[l] fp32,
    y [B, n_out].  With skip the output layer reads [a_L | x].  Returns
    (p, loss, dWs, dbs)."""
    B = x.shape[0]
    L = len(Ws) - 1
    acts, zs = [x], []
    a = x
    for l in range(L):
        z = a @ Ws[l].T + bs[l]
        zs.append(bf16(z))
        a = bf16(gelu(z))
        acts.append(a)
    H = a.shape[1]
    if skip:
        acts[L] = np.concatenate([a, x], axis=1)
    p = acts[L] @ Ws[L].T + bs[L]
    d = p[:, :n_out] - y
    scale = 1.0 / (B * n_out)
    loss = float((d * d).sum() * scale)
    g = np.zeros_like(p)
    g[:, :n_out] = 2.0 * d * scale
    g = bf16(g)
    dWs, dbs = [None] * (L + 1), [None] * (L + 1)
    for l in range(L, -1, -1):
        dWs[l] = g.T @ acts[l]
        dbs[l] = g.sum(0)
        if l > 0:
            Wh = Ws[l][:, :H] if (skip and l == L) else Ws[l]
            g = bf16((g @ Wh) * gelu_grad(zs[l - 1]))
    return p, loss, dWs, dbs
