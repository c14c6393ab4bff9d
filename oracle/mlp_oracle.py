"""CPU oracle of the warm-start surrogate (test infrastructure only).

A numpy restatement of the network the library trains on the GPU
(euler3d_b200/csrc/surrogate.cu): 6 -> 128 -> 128 -> 128 -> 5, exact-erf GELU
after the hidden layers, flat parameter layout W1 [128][16], b1 [128],
W2 [128][128], b2, W3 [128][128], b3, W4 [8][128], b4 [8] (padding rows and
columns zero).  With ``bf16=True`` it rounds at the same points as the GPU
kernels (weights, standardised inputs, hidden activations and back-propagated
hidden gradients to BF16, round to nearest even); sums are in FP64 here and
FP32 on the GPU, so the two agree to BF16 rounding of a few tie cases, not bit
for bit.  With ``bf16=False`` it is plain FP64 and is pinned against central
finite differences by the tests.  The reference solver has no counterpart of
this network; the oracle checks the project's own kernels.
"""
from __future__ import annotations

import math

import numpy as np

IN, H, OUT, N_IN, N_OUT = 16, 128, 8, 6, 5
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + OUT * H
N_PARAM = OFF_B4 + OUT

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to BF16 (nearest, ties to even); returns float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(a.shape)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3].reshape(H, H), p[OFF_B3:OFF_W4], p[OFF_W4:OFF_B4].reshape(OUT, H), p[OFF_B4:N_PARAM])


def wfree(mach, aoa_deg, gamma):
    a = np.radians(aoa_deg)
    q = mach * np.sqrt(gamma)
    u, v = q * np.cos(a), q * np.sin(a)
    z = np.zeros_like(u)
    return np.stack([np.ones_like(u), u, v, z, 0.5 * (u * u + v * v) + 1.0 / (gamma - 1.0)], axis=1)


def prepare(feat6, states5, norm, gamma, bf=True):
    """Standardised inputs [n][16] and scaled targets [n][5]."""
    f = np.asarray(feat6, dtype=np.float32)
    nm = np.asarray(norm, dtype=np.float32)
    x = np.zeros((f.shape[0], IN), dtype=np.float32)
    x[:, :N_IN] = (f[:, :N_IN] - nm[:N_IN]) / nm[8:8 + N_IN]
    if bf:
        x = bf16(x)
    t = None
    if states5 is not None:
        wf = wfree(f[:, 4].astype(np.float64), f[:, 5].astype(np.float64), gamma)
        t = (np.asarray(states5, dtype=np.float64) - wf) / nm[16:16 + N_OUT].astype(np.float64)
    return x.astype(np.float64), t


def forward(p, x, bf=True):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    q = (lambda a: bf16(a).astype(np.float64)) if bf else (lambda a: a)
    z1 = x @ q(W1).T + b1
    a1 = q(gelu(z1))
    z2 = a1 @ q(W2).T + b2
    a2 = q(gelu(z2))
    z3 = a2 @ q(W3).T + b3
    a3 = q(gelu(z3))
    y = a3 @ q(W4).T + b4
    return y[:, :N_OUT], (x, z1, a1, z2, a2, z3, a3)


def loss_and_grad(p, x, t, bf=True):
    """Mean squared error over rows and the 5 outputs, and its gradient (flat)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    q = (lambda a: bf16(a).astype(np.float64)) if bf else (lambda a: a)
    y, (x, z1, a1, z2, a2, z3, a3) = forward(p, x, bf)
    n = x.shape[0]
    e = y - t
    loss = float(np.mean(e * e))
    d4 = np.zeros((n, OUT))
    d4[:, :N_OUT] = 2.0 * e / (n * N_OUT)
    g = np.zeros(N_PARAM)
    g[OFF_W4:OFF_B4] = (d4.T @ a3).ravel()
    g[OFF_B4:N_PARAM] = d4.sum(axis=0)
    g3 = q((d4 @ q(W4)) * gelu_d(z3))
    g[OFF_W3:OFF_B3] = (g3.T @ a2).ravel()
    g[OFF_B3:OFF_W4] = g3.sum(axis=0)
    g2 = q((g3 @ q(W3)) * gelu_d(z2))
    g[OFF_W2:OFF_B2] = (g2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = g2.sum(axis=0)
    g1 = q((g2 @ q(W2)) * gelu_d(z1))
    g[OFF_W1:OFF_B1] = (g1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = g1.sum(axis=0)
    return loss, g


def predict(p, feat6, norm, gamma, bf=True):
    x, _ = prepare(feat6, None, norm, gamma, bf)
    y, _ = forward(p, x, bf)
    f = np.asarray(feat6, dtype=np.float64)
    wf = wfree(f[:, 4], f[:, 5], gamma)
    return wf + np.asarray(norm, dtype=np.float64)[16:16 + N_OUT] * y
