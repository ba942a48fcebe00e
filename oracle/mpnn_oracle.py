"""CPU restatement (numpy, FP64) of the learned correction's network: the
forward pass and the gradient of its training loss. The network has no
reference counterpart; this restatement is the checker of the GPU forward
and backward kernels (fvm_b200/csrc/learned.cu), and its own gradient is
checked by finite differences.

TEST INFRASTRUCTURE ONLY -- imported by tests/ as the checker. The product
(fvm_b200) never imports it.

Graph: a CSR matrix with implicit diagonal (row, col, diag, off) over n
nodes; w_ij = |a_ij| / |a_ii| on every stored entry. Parameter layout (6337
floats): encoder weight [0:32] and bias [32:64]; layer l (l = 0, 1, 2) at
64 + 2080 l: Ws (32 x 32, row = output channel), Wm (32 x 32), b (32);
decoder weight [6304:6336] and bias [6336].
"""
from __future__ import annotations

import numpy as np

W = 32
LAYERS = 3
LAYER = 2 * W * W + W
DEC_W = 64 + LAYERS * LAYER
N_PARAMS = DEC_W + W + 1


def _coupling(row, col, diag, off):
    """Sparse n x n matrix of the couplings w_ij (duplicates summed)."""
    from scipy.sparse import csr_matrix

    n = len(diag)
    rid = np.repeat(np.arange(n), np.diff(row))
    w = np.abs(off) / np.abs(diag[rid])
    return csr_matrix((w, (rid, np.asarray(col))), shape=(n, n))


def _unpack(P):
    P = np.asarray(P, dtype=np.float64)
    layers = []
    for l in range(LAYERS):
        o = 64 + l * LAYER
        layers.append((P[o: o + W * W].reshape(W, W), P[o + W * W: o + 2 * W * W].reshape(W, W),
                       P[o + 2 * W * W: o + LAYER]))
    return P[0:W], P[W:2 * W], layers, P[DEC_W: DEC_W + W], P[DEC_W + W]


def forward(P, row, col, diag, off, r, keep=False):
    """Correction d = s * (decoder(h3)) for residual r."""
    Wc = _coupling(row, col, diag, off)
    we, be, layers, wd, bd = _unpack(P)
    d = np.abs(diag)
    s = float(np.mean(np.abs(r) / d))
    u = r / (d * s) if s > 0 else np.zeros_like(r)
    z0 = u[:, None] * we[None, :] + be[None, :]
    H = [np.maximum(z0, 0.0)]
    Z, M = [z0], []
    for Ws, Wm, b in layers:
        m = Wc @ H[-1]
        z = H[-1] @ Ws.T + m @ Wm.T + b[None, :]
        M.append(m)
        Z.append(z)
        H.append(np.maximum(z, 0.0))
    y = H[-1] @ wd + bd
    out = s * y
    if keep:
        return out, dict(Wc=Wc, u=u, s=s, H=H, Z=Z, M=M, layers=layers, wd=wd)
    return out


def loss_and_gradient(P, row, col, diag, off, r, e):
    """Relative squared error sum (d - e)^2 / sum e^2 and its gradient."""
    out, c = forward(P, row, col, diag, off, r, keep=True)
    E2 = float(np.sum(e * e)) or 1.0
    diff = out - e
    loss = float(np.sum(diff * diff) / E2)
    g = np.zeros(N_PARAMS)
    gy = 2.0 * c["s"] * diff / E2
    g[DEC_W: DEC_W + W] = c["H"][-1].T @ gy
    g[DEC_W + W] = gy.sum()
    dH = gy[:, None] * c["wd"][None, :]
    for l in range(LAYERS - 1, -1, -1):
        Ws, Wm, b = c["layers"][l]
        dz = dH * (c["Z"][l + 1] > 0)
        o = 64 + l * LAYER
        g[o: o + W * W] = (dz.T @ c["H"][l]).ravel()
        g[o + W * W: o + 2 * W * W] = (dz.T @ c["M"][l]).ravel()
        g[o + 2 * W * W: o + LAYER] = dz.sum(axis=0)
        dH = dz @ Ws + c["Wc"].T @ (dz @ Wm)
    dz0 = dH * (c["Z"][0] > 0)
    g[0:W] = dz0.T @ c["u"]
    g[W:2 * W] = dz0.sum(axis=0)
    return loss, g
