"""numpy restatement of the learned warm-start network (CPU oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  The network has no
counterpart in the spectral-init crate; it predicts the starting block of the
crate's LOBPCG (``src/solvers/lobpcg.rs:227-465``), whose random start it
replaces.  This module restates the device forward and backward passes so the
GPU gradients can be checked, and it is itself checked against central finite
differences (``rounding=False``).

Network (hidden 64, [H | Ahat H] concatenation, ReLU, output 16 columns):
    A_l   = [H_l | Ahat H_l]                Ahat = -offdiag(L) = D^-1/2 W D^-1/2
    H_l+1 = ReLU(A_l Wt_l^T + b_l)          l = 0, 1, 2
    Y     = A_3 Wt_out^T + b_out
Loss: L = 1 - tr(G^-1 M) / k with G = Y^T Y, C = V^T Y, M = C^T C over the
first k columns of Y.  With ``rounding=True`` the values the device stores in
bf16 (weights, activations, dY, dZ) are rounded the same way.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

HIDDEN, CAT, OUT, LAYERS, FEATURES = 64, 128, 16, 3, 5


def param_count() -> int:
    return LAYERS * (HIDDEN * CAT + HIDDEN) + OUT * CAT + OUT


def unpack(p: np.ndarray):
    """Flat parameter vector -> [(Wt_l [64 x 128], b_l)], (Wt_out [16 x 128], b_out)."""
    p = np.asarray(p, dtype=np.float32)
    layers, o = [], 0
    for _ in range(LAYERS):
        wt = p[o:o + HIDDEN * CAT].reshape(HIDDEN, CAT)
        o += HIDDEN * CAT
        layers.append((wt, p[o:o + HIDDEN]))
        o += HIDDEN
    wt = p[o:o + OUT * CAT].reshape(OUT, CAT)
    o += OUT * CAT
    return layers, (wt, p[o:o + OUT])


def pack(layer_grads, out_grad) -> np.ndarray:
    parts = []
    for gw, gb in layer_grads:
        parts += [np.asarray(gw).ravel(), np.asarray(gb).ravel()]
    parts += [np.asarray(out_grad[0]).ravel(), np.asarray(out_grad[1]).ravel()]
    return np.concatenate(parts)


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def ahat_from_values(indptr, indices, values_f32, n) -> sp.csr_matrix:
    """Ahat = -V for an implicit-unit-diagonal Laplacian with off-diagonal values V."""
    v = -np.asarray(values_f32, dtype=np.float32).astype(np.float64)
    return sp.csr_matrix((v, np.asarray(indices), np.asarray(indptr)), shape=(n, n))


def forward(params, ahat: sp.csr_matrix, features: np.ndarray, rounding: bool = True):
    """Returns (Y [n x 16] f64, cache)."""
    rnd = bf16 if rounding else (lambda z: np.asarray(z, dtype=np.float64))
    layers, (wto, bo) = unpack(params)
    n = features.shape[0]
    h = np.zeros((n, HIDDEN))
    h[:, :FEATURES] = np.asarray(features, dtype=np.float32)
    h = rnd(h)
    acts = []
    for l in range(LAYERS + 1):
        a = np.hstack([h, rnd(ahat @ h)])
        acts.append(a)
        if l < LAYERS:
            wt, b = layers[l]
            z = a @ rnd(wt).T + b.astype(np.float64)
            h = rnd(np.maximum(z, 0.0))
    y = acts[-1] @ rnd(wto).T + bo.astype(np.float64)
    return y, {"acts": acts, "rnd": rnd}


def loss_and_dy(y: np.ndarray, v: np.ndarray, k: int):
    yk = y[:, :k]
    g = yk.T @ yk
    c = v[:, :k].T @ yk
    m = c.T @ c
    gi = np.linalg.inv(g)
    loss = 1.0 - np.trace(gi @ m) / k
    dy = np.zeros_like(y)
    dy[:, :k] = -(2.0 / k) * (v[:, :k] @ (c @ gi) - yk @ (gi @ m @ gi))
    return loss, dy


def backward(params, ahat: sp.csr_matrix, cache, dy: np.ndarray) -> np.ndarray:
    """Flat gradient (same layout as the parameters) from dL/dY."""
    rnd = cache["rnd"]
    acts = cache["acts"]
    layers, (wto, _) = unpack(params)
    dy = rnd(dy)
    a3 = acts[LAYERS]
    g_out = ((a3.T @ dy).T, dy.sum(axis=0))
    da = dy @ rnd(wto)                                    # [n x 128]
    grads = [None] * LAYERS
    for l in range(LAYERS - 1, -1, -1):
        h_next = acts[l + 1][:, :HIDDEN]
        dh = da[:, :HIDDEN] + ahat @ da[:, HIDDEN:]        # Ahat symmetric
        dz = rnd(dh * (h_next > 0))
        grads[l] = ((acts[l].T @ dz).T, dz.sum(axis=0))
        if l > 0:
            da = dz @ rnd(layers[l][0])
    return pack(grads, g_out)


def loss_and_grad(params, ahat, features, v, k, rounding=True):
    y, cache = forward(params, ahat, features, rounding)
    loss, dy = loss_and_dy(y, v, k)
    return loss, backward(params, ahat, cache, dy)
