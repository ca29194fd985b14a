"""CPU oracle of the learned trajectory-length scheduler's CNN -- TEST
INFRASTRUCTURE ONLY (used by ``tests/`` as the checker of the GPU forward,
backward and inference kernels; never by the product path).

The network has no counterpart in the reference; this is a plain NumPy
restatement of its definition in float64, with the same bfloat16 roundings
as the device (inputs, weights, hidden activations, and the gradients where
they enter a product), straight-through in the backward pass:

    x1[s, t, f]  = bf16(uv[clamp(cx-8+4ti+di), clamp(cy-8+4tj+dj), c]),
                   t = 4ti+tj, f = 2(4di+dj)+c, (cx, cy) = seed pixel + pad
    a1 = bf16(relu(x1 @ w1 + b1))                    [s, 16, 32]
    x2[s, u, g]  = a1[s, 4(2ui+ei) + 2uj+ej, o],     u = 2ui+uj, g = 32(2ei+ej)+o
    a2 = bf16(relu(x2 @ w2 + b2))                    [s, 4, 64]
    y  = a2.reshape(s, 256) @ w3 + b3                [s, 2]
    loss = mean((y - t)^2) over all s and both outputs
"""
from __future__ import annotations

import numpy as np

SHAPES = (("w1", (32, 32)), ("b1", (32,)), ("w2", (128, 64)), ("b2", (64,)),
          ("w3", (256, 2)), ("b3", (2,)))


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even); NaN-free inputs."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(np.shape(x))


def gather(uv, pad, seeds, index=None):
    """x1 [n, 16, 32] (bfloat16 values as float64) for seeds [n or index]."""
    nxp, nyp = uv.shape[:2]
    s = seeds if index is None else seeds[np.asarray(index, np.int64)]
    cx = s[:, 0].astype(np.int64) + pad
    cy = s[:, 1].astype(np.int64) + pad
    t = np.arange(16)
    m = np.arange(16)
    ti, tj = t // 4, t % 4
    di, dj = m // 4, m % 4
    x = cx[:, None, None] - 8 + 4 * ti[None, :, None] + di[None, None, :]
    y = cy[:, None, None] - 8 + 4 * tj[None, :, None] + dj[None, None, :]
    x = np.clip(x, 0, nxp - 1)
    y = np.clip(y, 0, nyp - 1)
    v = bf16(uv[x, y, :])  # [n, 16 tiles, 16 cells, 2]
    return v.reshape(s.shape[0], 16, 32).astype(np.float64)


_T2 = np.array([[4 * (2 * (u >> 1) + (g >> 6)) + 2 * (u & 1) + ((g >> 5) & 1) for g in range(128)]
                for u in range(4)])
_O2 = np.array([[g & 31 for g in range(128)] for _ in range(4)])


def _rearrange(a1):
    """a1 [n, 16, 32] -> x2 [n, 4, 128]"""
    return a1[:, _T2, _O2]


def _rearrange_back(dx2):
    n = dx2.shape[0]
    da1 = np.zeros((n, 16, 32))
    np.add.at(da1, (slice(None), _T2, _O2), dx2)
    return da1


def forward(w, x1, rounding=True):
    r = bf16 if rounding else (lambda a: a)
    W = {k: (r(np.asarray(v, np.float32)).astype(np.float64) if rounding else np.asarray(v, np.float64))
         for k, v in w.items()}
    z1 = x1 @ W["w1"] + W["b1"]
    a1 = np.maximum(z1, 0.0)
    a1 = r(a1.astype(np.float32)).astype(np.float64) if rounding else a1
    x2 = _rearrange(a1)
    z2 = x2 @ W["w2"] + W["b2"]
    a2 = np.maximum(z2, 0.0)
    a2 = r(a2.astype(np.float32)).astype(np.float64) if rounding else a2
    x3 = a2.reshape(x1.shape[0], 256)
    y = x3 @ W["w3"] + W["b3"]
    return y, dict(W=W, z1=z1, x2=x2, z2=z2, x3=x3)


def loss_and_grad(w, x1, target, rounding=True):
    """Mean-squared-error loss and its gradients w.r.t. every weight."""
    y, c = forward(w, x1, rounding)
    n_el = y.size
    d = y - target
    loss = float((d * d).sum() / n_el)
    dy = 2.0 * d / n_el
    W = c["W"]
    # every GEMM operand is bfloat16 (the tensor cores' input type): the
    # gradients are rounded where they enter a product, the bias gradients
    # sum them unrounded
    r = (lambda a: bf16(a.astype(np.float32)).astype(np.float64)) if rounding else (lambda a: a)
    g = {"w3": c["x3"].T @ r(dy), "b3": dy.sum(0)}
    dz2 = (r(dy) @ W["w3"].T).reshape(-1, 4, 64) * (c["z2"] > 0)
    g["w2"] = c["x2"].reshape(-1, 128).T @ r(dz2.reshape(-1, 64))
    g["b2"] = dz2.reshape(-1, 64).sum(0)
    dz1 = _rearrange_back((r(dz2.reshape(-1, 64)) @ W["w2"].T).reshape(-1, 4, 128)) * (c["z1"] > 0)
    g["w1"] = x1.reshape(-1, 32).T @ r(dz1.reshape(-1, 32))
    g["b1"] = dz1.reshape(-1, 32).sum(0)
    return loss, g


def predict(w, uv, pad, seeds):
    return forward(w, gather(uv, pad, seeds))[0]
