"""CPU restatement of the learned start-distance proposal's network.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the device
forward / backward / feature kernels.  The reference has no learned
component, so this restates the network as the product specifies it:

    x (80 features) -> GELU(W1 x + b1) -> GELU(W2 . + b2) -> GELU(W3 . + b3)
                    -> wo . + bo = predicted log(first-hit t)

GELU is the tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
(Hendrycks & Gimpel, "Gaussian Error Linear Units", 2016).  The loss of a
batch is the mean squared error against log t.  Everything is float64.

Flat parameter layout (VX_MLP_FLOATS = 13569 f32): W1[64][80] (columns
70..79 zero), b1[64], W2[64][64], b2[64], W3[64][64], b3[64], wo[64], bo.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 80, 64
SIZES = [("W1", (N_H, N_IN)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
         ("W3", (N_H, N_H)), ("b3", (N_H,)), ("wo", (N_H,)), ("bo", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)
assert N_PARAMS == 13569
K0, K1 = np.sqrt(2.0 / np.pi), 0.044715


def unpack(flat: np.ndarray) -> dict:
    flat = np.asarray(flat, np.float64)
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SIZES])


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z):
    th = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1.0 + th) + 0.5 * z * (1.0 - th * th) * K0 * (1.0 + 3.0 * K1 * z * z)


def forward(flat: np.ndarray, X: np.ndarray):
    """Predicted log t per row of X (n x 80) and the layer cache."""
    P = unpack(flat)
    X = np.asarray(X, np.float64)
    z1 = X @ P["W1"].T + P["b1"]
    a1 = gelu(z1)
    z2 = a1 @ P["W2"].T + P["b2"]
    a2 = gelu(z2)
    z3 = a2 @ P["W3"].T + P["b3"]
    a3 = gelu(z3)
    y = a3 @ P["wo"] + P["bo"][0]
    return y, (X, z1, a1, z2, a2, z3, a3)


def loss_and_grad(flat: np.ndarray, X: np.ndarray, target: np.ndarray):
    """Mean squared error of log t and its gradient (flat layout)."""
    P = unpack(flat)
    y, (X, z1, a1, z2, a2, z3, a3) = forward(flat, X)
    B = X.shape[0]
    e = y - np.asarray(target, np.float64)
    loss = float(np.mean(e * e))
    dy = 2.0 * e / B
    g = {"wo": a3.T @ dy, "bo": np.array([dy.sum()])}
    dz3 = np.outer(dy, P["wo"]) * gelu_grad(z3)
    g["W3"], g["b3"] = dz3.T @ a2, dz3.sum(0)
    dz2 = (dz3 @ P["W3"]) * gelu_grad(z2)
    g["W2"], g["b2"] = dz2.T @ a1, dz2.sum(0)
    dz1 = (dz2 @ P["W2"]) * gelu_grad(z1)
    g["W1"], g["b1"] = dz1.T @ X, dz1.sum(0)
    return loss, pack(g)


def features(org: np.ndarray, dirs: np.ndarray, chunk_words: np.ndarray) -> np.ndarray:
    """Feature rows: origin mod 64 / 64, direction, the 64 tile bits of the
    chunk holding the origin (given per ray), zero padding."""
    org = np.asarray(org, np.float32)
    f = np.zeros((org.shape[0], N_IN), np.float32)
    f[:, 0:3] = (org - np.float32(64.0) * np.floor(org * np.float32(1.0 / 64.0))) * np.float32(1.0 / 64.0)
    f[:, 3:6] = dirs
    w = np.asarray(chunk_words, np.uint64)
    bits = (w[:, None] >> np.arange(64, dtype=np.uint64)[None, :]) & np.uint64(1)
    f[:, 6:70] = bits.astype(np.float32)
    return f


def origin_chunk_words(chunk_mask: np.ndarray, dims_bricks, org: np.ndarray,
                       window=(0, 0, 0)) -> np.ndarray:
    """Tile bits of the chunk holding each origin (slot coordinates, x/z
    folded into the window), 0 for an origin outside the window."""
    bx, by, bz = dims_bricks
    vx, vy, vz = bx * 4, by * 4, bz * 4
    cx, cy = (bx // 4 + 3) // 4, (by // 4 + 3) // 4
    v = np.floor(np.asarray(org, np.float32)).astype(np.int64)
    rel = v - np.asarray(window, np.int64)[None, :]
    inside = ((rel[:, 0] >= 0) & (rel[:, 0] < vx) & (rel[:, 1] >= 0) & (rel[:, 1] < vy) &
              (rel[:, 2] >= 0) & (rel[:, 2] < vz) & (v[:, 1] >= 0) & (v[:, 1] < vy))
    sx, sz = np.mod(v[:, 0], vx), np.mod(v[:, 2], vz)
    ci = (sx >> 6) + (np.clip(v[:, 1], 0, vy - 1) >> 6) * cx + (sz >> 6) * cx * cy
    return np.where(inside, chunk_mask[ci], np.uint64(0)).astype(np.uint64)
