"""Float64 restatement of the transmittance network (TEST INFRASTRUCTURE ONLY).

Same architecture, parameter layout and rounding points as the library's
training kernels: inputs, weights and post-ReLU activations are rounded to
bfloat16 before they enter a product; products and sums are float64 here
(float32 on the device). The backward pass treats the roundings as identity.
Used to check the device gradients and the input encoding."""
from __future__ import annotations

import numpy as np

K_IN, K_USED, K_HID, K_FREQ = 112, 102, 64, 16
OFF = {}
_o = 0
for name, size in [("W1", K_IN * K_HID), ("B1", K_HID), ("W2", K_HID * K_HID), ("B2", K_HID),
                   ("W3", K_HID * K_HID), ("B3", K_HID), ("W4", K_HID * K_HID), ("B4", K_HID),
                   ("W5", K_HID), ("B5", 1)]:
    OFF[name] = (_o, size)
    _o += size
N_PARAMS = _o


def bf16(x):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, np.float64)
    g = lambda k: P[OFF[k][0]:OFF[k][0] + OFF[k][1]]  # noqa: E731
    W = [g("W1").reshape(K_IN, K_HID)] + [g(f"W{i}").reshape(K_HID, K_HID) for i in (2, 3, 4)]
    B = [g(f"B{i}") for i in (1, 2, 3, 4)]
    return W, B, g("W5"), g("B5")[0]


def encode(pos, lfeat, bmin, bmax):
    """Input encoding (float64): [u*2-1, light, sin/cos(pi f_k u_a), zeros]."""
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    u = (pos - np.asarray(bmin)) / (np.asarray(bmax) - np.asarray(bmin))
    n = pos.shape[0]
    X = np.zeros((n, K_IN))
    X[:, 0:3] = u * 2 - 1
    X[:, 3:6] = np.asarray(lfeat, np.float64).reshape(-1, 3)
    f = 2.0 ** (7.0 * np.arange(K_FREQ) / 15.0)
    for a in range(3):
        ang = np.pi * f[None, :] * u[:, a:a + 1]
        X[:, 6 + a * 32:6 + a * 32 + 32:2] = np.sin(ang)
        X[:, 7 + a * 32:6 + a * 32 + 32:2] = np.cos(ang)
    return X


def forward_backward(P, X, target):
    """Returns (loss, grad, T) for features X (n x 112) and targets."""
    W, B, w5, b5 = unpack(P)
    Wb = [bf16(w) for w in W]
    w5b = bf16(w5)
    n = X.shape[0]
    hs = [bf16(X)]
    for l in range(4):
        z = hs[-1] @ Wb[l] + B[l]
        hs.append(bf16(np.maximum(z, 0.0)))
    zz = hs[4] @ w5b + b5
    T = 1.0 / (1.0 + np.exp(-zz))
    d = T - np.asarray(target, np.float64)
    loss = np.mean(d * d)
    dz = (2.0 / n) * d * T * (1 - T)
    grad = np.zeros(N_PARAMS)
    grad[OFF["W5"][0]:OFF["W5"][0] + K_HID] = hs[4].T @ dz
    grad[OFF["B5"][0]] = dz.sum()
    dh = np.outer(dz, w5b) * (hs[4] > 0)
    for l in (3, 2, 1, 0):
        o, sz = OFF[f"W{l + 1}"]
        grad[o:o + sz] = (hs[l].T @ dh).ravel()
        o, sz = OFF[f"B{l + 1}"]
        grad[o:o + sz] = dh.sum(axis=0)
        if l > 0:
            dh = (dh @ Wb[l].T) * (hs[l] > 0)
    return loss, grad, T
