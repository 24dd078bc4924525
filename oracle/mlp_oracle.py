"""CPU restatement (numpy; test infrastructure) of the learned warm-start MLP of
project_superdex_b200/csrc/sdx_mlp.cu: forward with BF16-rounded inputs, weights and hidden activations
(FP32 products and sums), the mean-squared-error loss and its gradients, and Adam. The reference has no
such network (its mochi_core/include/mochi_core/ai/mlp.h is CPU inference only), so this restatement is
the checker for the GPU forward / backward kernels.

Parameter layout (flat FP32 vector): W1 128x16, b1 128, W2 128x128, b2 128, W3 128x128, b3 128,
W4 16x128 (rows 0..2 used), b4 16 (0..2 used).
"""
from __future__ import annotations

import numpy as np
from math import erf, sqrt

N_PARAMS = 37264
OFF = {"W1": (0, (128, 16)), "b1": (2048, (128,)), "W2": (2176, (128, 128)), "b2": (18560, (128,)),
       "W3": (18688, (128, 128)), "b3": (35072, (128,)), "W4": (35200, (16, 128)), "b4": (37248, (16,))}

_verf = np.vectorize(erf)


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p):
    return {k: np.asarray(p[o:o + int(np.prod(s))], np.float32).reshape(s) for k, (o, s) in OFF.items()}


def gelu(z):
    return 0.5 * z * (1.0 + _verf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _verf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * np.pi)


def forward(p, X, keep=False):
    P = unpack(p)
    Xb = bf16(X).astype(np.float64)
    W = [bf16(P["W1"]).astype(np.float64), bf16(P["W2"]).astype(np.float64), bf16(P["W3"]).astype(np.float64),
         bf16(P["W4"]).astype(np.float64)]
    b = [P["b1"], P["b2"], P["b3"], P["b4"]]
    h = Xb
    Zs, Hs = [], [Xb]
    for l in range(3):
        z = h @ W[l].T + b[l]
        Zs.append(z)
        h = bf16(gelu(z).astype(np.float32)).astype(np.float64)
        Hs.append(h)
    y = (h @ W[3].T + b[3])[:, :3]
    if keep:
        return y, Zs, Hs, W
    return y


def loss_and_grad(p, X, T):
    """MSE over the 3 outputs and all samples, and its gradient (straight-through the BF16 rounding)."""
    y, Zs, Hs, W = forward(p, X, keep=True)
    n = X.shape[0]
    d = y - T
    loss = float(np.mean(d * d))
    dY = 2.0 * d / (3.0 * n)
    g = np.zeros(N_PARAMS)
    o, s = OFF["W4"]
    gW4 = np.zeros((16, 128))
    gW4[:3] = dY.T @ Hs[3]
    g[o:o + gW4.size] = gW4.reshape(-1)
    g[OFF["b4"][0]:OFF["b4"][0] + 3] = dY.sum(0)
    dH = dY @ W[3][:3]
    for l in (2, 1, 0):
        dZ = dH * gelu_grad(Zs[l])
        wname, bname = f"W{l + 1}", f"b{l + 1}"
        gw = dZ.T @ Hs[l]
        if l == 0:
            gw[:, 15] = 0.0
        g[OFF[wname][0]:OFF[wname][0] + gw.size] = gw.reshape(-1)
        g[OFF[bname][0]:OFF[bname][0] + 128] = dZ.sum(0)
        dH = dZ @ W[l]
    return loss, g
