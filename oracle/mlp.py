"""TEST INFRASTRUCTURE ONLY: a NumPy restatement of the learned
initialiser's network and loss (forward and hand-derived backward), the
checker for the library's BF16 tensor-core kernels (ocpf_mlp_forward /
ocpf_mlp_grad). No counterpart in the reference.

Layout as in include/ocp_flash.h: one FP32 parameter vector
W1[64][16] b1[64] W2[64][64] b2[64] W3[16][64] b3[16]; inputs x[f, s].

With ``bf16=True`` it rounds to bfloat16 (round to nearest even) exactly
where the kernels do -- the GEMM operands (inputs, weights, hidden
activations, back-propagated deltas) -- and accumulates in float64, so it
differs from the kernels only by FP32 accumulation order. With
``bf16=False`` it is the plain float64 network, which finite differences
check.
"""
from __future__ import annotations

import numpy as np

H, IO = 64, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IO
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + IO * H
NPARAM = OFF_B3 + IO


def bf16_round(a):
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IO), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(IO, H), p[OFF_B3:NPARAM])


def _silu(v):
    return v / (1 + np.exp(-v))


def _silu_grad(v):
    s = 1 / (1 + np.exp(-v))
    return s * (1 + v * (1 - s))


def forward(p, x, bf16=True):
    """Outputs [16, n] (rows beyond nout are the padding's outputs)."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(p)
    nin, n = x.shape
    X = np.zeros((IO, n))
    X[:nin] = x
    a1 = r(W1) @ r(X) + b1[:, None]
    h1 = r(_silu(a1))
    a2 = r(W2) @ h1 + b2[:, None]
    h2 = r(_silu(a2))
    return r(W3) @ h2 + b3[:, None], (X, a1, h1, a2, h2)


def loss_and_grad(p, x, t, w, lnk_weight=1.0, bf16=True):
    """(loss sums [logistic, ln K], gradient of the mean loss) for
    x [nin, n], t [nout, n], w [n]."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(p)
    nout, n = t.shape
    out, (X, a1, h1, a2, h2) = forward(p, x, bf16)
    z = out[0]
    y = t[0]
    bce = np.sum(np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - y * z)
    e = out[1:nout] - t[1:]
    mse = np.sum(w * np.sum(e * e, axis=0) / (nout - 1))
    d3 = np.zeros((IO, n))
    d3[0] = (1 / (1 + np.exp(-z)) - y) / n
    d3[1:nout] = 2 * w * lnk_weight / (nout - 1) * e / n
    d3 = r(d3)
    d2 = r((r(W3).T @ d3) * _silu_grad(a2))
    d1 = r((r(W2).T @ d2) * _silu_grad(a1))
    g = np.zeros(NPARAM)
    g[OFF_W1:OFF_B1] = (d1 @ r(X).T).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(axis=1)
    g[OFF_W2:OFF_B2] = (d2 @ h1.T).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(axis=1)
    g[OFF_W3:OFF_B3] = (d3 @ h2.T).ravel()
    g[OFF_B3:NPARAM] = d3.sum(axis=1)
    return np.array([bce, mse]), g
