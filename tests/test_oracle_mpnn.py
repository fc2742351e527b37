"""The warm-start network's CPU oracle against central finite differences.

The oracle's analytic backward pass (``oracle/mpnn_oracle.py``) is what the
device gradients are checked against, so it is pinned here first: without
bf16 rounding, every sampled partial derivative must match a central
difference of the loss.
"""
import numpy as np
import scipy.sparse as sp

from oracle import mpnn_oracle as M


def _tiny_problem(seed=0, n=40, k=3):
    rng = np.random.default_rng(seed)
    w = sp.random(n, n, density=0.15, random_state=seed, data_rvs=lambda s: rng.uniform(0.1, 1.0, s))
    w = sp.csr_matrix(w + w.T)
    w.setdiag(0)
    w.eliminate_zeros()
    w = w + sp.eye(n, k=1) + sp.eye(n, k=-1)       # connected
    d = np.asarray(w.sum(axis=1)).ravel()
    dinv = sp.diags(1.0 / np.sqrt(d))
    ahat = sp.csr_matrix(dinv @ w @ dinv)
    lap = np.eye(n) - ahat.toarray()
    _, vecs = np.linalg.eigh(lap)
    feats = rng.standard_normal((n, M.FEATURES)).astype(np.float32)
    params = (rng.standard_normal(M.param_count()) * 0.15).astype(np.float32).astype(np.float64)
    return ahat, feats, vecs[:, :k], params, k


def test_param_layout_round_trip():
    p = np.arange(M.param_count(), dtype=np.float64)
    layers, out = M.unpack(p)
    q = M.pack([(w, b) for w, b in layers], out)
    assert np.array_equal(p.astype(np.float32), q)
    assert M.param_count() == 26832


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even
    assert r[2] == 1.0 + 2 ** -6                  # tie to even (upwards)
    assert r[3] == -2.5
    assert abs(r[4] - 1e-3) <= 2 ** -8 * 1e-3


def test_oracle_gradient_matches_finite_differences():
    ahat, feats, v, params, k = _tiny_problem()
    loss, grad = M.loss_and_grad(params, ahat, feats, v, k, rounding=False)
    assert 0.0 <= loss <= 1.0
    rng = np.random.default_rng(1)
    idx = rng.choice(M.param_count(), size=60, replace=False)
    # include a few biases and output weights
    idx = np.concatenate([idx, [M.param_count() - 1, M.param_count() - 20, 8192 + 3]])
    eps = 1e-5
    for i in idx:
        p1 = params.copy()
        p2 = params.copy()
        p1[i] += eps
        p2[i] -= eps
        # unpack() works in float32: perturb through a float64-preserving path
        l1 = _loss64(p1, ahat, feats, v, k)
        l2 = _loss64(p2, ahat, feats, v, k)
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-4 * max(1.0, abs(fd)) + 1e-6, (i, fd, grad[i])


def _loss64(p, ahat, feats, v, k):
    """Loss with float64 parameters (the oracle's unpack rounds to float32)."""
    layers, o = [], 0
    for _ in range(M.LAYERS):
        wt = p[o:o + M.HIDDEN * M.CAT].reshape(M.HIDDEN, M.CAT)
        o += M.HIDDEN * M.CAT
        layers.append((wt, p[o:o + M.HIDDEN]))
        o += M.HIDDEN
    wto = p[o:o + M.OUT * M.CAT].reshape(M.OUT, M.CAT)
    o += M.OUT * M.CAT
    bo = p[o:o + M.OUT]
    n = feats.shape[0]
    h = np.zeros((n, M.HIDDEN))
    h[:, :M.FEATURES] = feats
    for l in range(M.LAYERS):
        a = np.hstack([h, ahat @ h])
        h = np.maximum(a @ layers[l][0].T + layers[l][1], 0.0)
    a = np.hstack([h, ahat @ h])
    y = a @ wto.T + bo
    return M.loss_and_dy(y, v, k)[0]
