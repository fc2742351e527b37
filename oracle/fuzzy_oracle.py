"""CPU restatement of the fuzzy-kNN graph construction that produces the
crate's input graphs: the oracle for the device kernels of
``si_fuzzy_graph`` (``csrc/fuzzy.cu``).

TEST INFRASTRUCTURE ONLY (the checker of ``tests/``; never the product path).

The crate consumes a UMAP fuzzy simplicial set; its fixture generator
(tests/generate_fixtures.py:70-182 of the reference) builds it in five stages:

1. exact kNN: the full Euclidean distance matrix with the diagonal excluded,
   rows sorted ascending, the first k kept (``:70-94``), distances as f32;
2. ``smooth_knn_dist`` of umap-learn 0.5.11 (an un-vendored dependency of the
   generator) on the f32 distances with k neighbours (``:97-113``);
3. ``compute_membership_strengths`` of umap-learn (``:116-142``);
4. the fuzzy union A + A^T - A∘A^T (``:145-161``);
5. pruning of entries below max / n_epochs, n_epochs = 500 for n <= 10000,
   else 200 (``:164-182``).

Stages 2 and 3 restate umap-learn's published algorithm (McInnes, Healy and
Melville, "UMAP", 2018, section 3 and its reference implementation): rho is
the distance to the nearest neighbour at a positive distance
(local connectivity 1); sigma is found by bisection (64 steps, tolerance
1e-5) so that sum over the neighbours after the first of
exp(-max(d - rho, 0) / sigma) equals log2(k); sigma is floored at 1e-3 times
the mean distance of the row (of all rows when rho = 0); the membership of
neighbour j of i is 1 when d_ij <= rho_i or sigma_i = 0, else
exp(-(d_ij - rho_i) / sigma_i).  The arithmetic follows the generator's
types: distances, rho and sigma are f32, the bisection runs in f64, the
membership exponential in f32.

One point is pinned by the fixtures rather than by the paper: when the sum at
the starting sigma = 1 is below log2(k), the fixtures hold sigma = +inf (85 of
the 200 rows of blobs_connected_200, exactly the rows whose root lies above
1; the others agree to f32 rounding).  The generator's bisection takes the
midpoint against an infinite upper bound instead of doubling, so such a row
keeps sigma = +inf and every membership of it is 1.  ``smooth_knn`` follows
that by default (``upward="midpoint"``); ``upward="double"`` is the doubling
search of the paper's implementation.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

SMOOTH_K_TOLERANCE = 1e-5
MIN_K_DIST_SCALE = 1e-3
N_ITER = 64


def knn_exact(x: np.ndarray, k: int):
    """Stage 1: (indices int32 [n, k], distances f32 [n, k]), self excluded,
    ascending by distance (stable among equal distances)."""
    x = np.asarray(x, dtype=np.float64)
    sq = (x * x).sum(1)
    d2 = sq[:, None] - 2.0 * (x @ x.T) + sq[None, :]
    d = np.sqrt(np.maximum(d2, 0.0))
    np.fill_diagonal(d, np.inf)
    order = np.argsort(d, axis=1, kind="stable")[:, :k]
    return order.astype(np.int32), np.take_along_axis(d, order, axis=1).astype(np.float32)


def smooth_knn(dists: np.ndarray, k: int, upward: str = "midpoint"):
    """Stage 2: (sigmas f32 [n], rhos f32 [n]) for f32 distances [n, k]."""
    assert upward in ("midpoint", "double")
    dists = np.asarray(dists, dtype=np.float32)
    n = dists.shape[0]
    target = math.log2(k)
    mean_all = float(np.mean(dists))
    sig = np.zeros(n, dtype=np.float32)
    rho = np.zeros(n, dtype=np.float32)
    for i in range(n):
        row = dists[i]
        pos = row[row > 0.0]
        if pos.shape[0] >= 1:
            rho[i] = pos[0]
        lo, hi, mid = 0.0, math.inf, 1.0
        for _ in range(N_ITER):
            psum = 0.0
            for j in range(1, row.shape[0]):
                dd = np.float32(row[j] - rho[i])
                psum += math.exp(-(float(dd) / mid)) if dd > 0 else 1.0
            if abs(psum - target) < SMOOTH_K_TOLERANCE:
                break
            if psum > target:
                hi = mid
                mid = (lo + hi) / 2.0
            else:
                lo = mid
                mid = mid * 2.0 if (hi == math.inf and upward == "double") else (lo + hi) / 2.0
        floor = MIN_K_DIST_SCALE * (float(np.mean(row)) if rho[i] > 0.0 else mean_all)
        sig[i] = floor if mid < floor else mid
    return sig, rho


def membership(knn_indices: np.ndarray, dists: np.ndarray, sigmas: np.ndarray, rhos: np.ndarray) -> sp.coo_matrix:
    """Stage 3: the directed membership graph (COO, f32; zeros removed)."""
    knn_indices = np.asarray(knn_indices, dtype=np.int64)
    dists = np.asarray(dists, dtype=np.float32)
    n, k = knn_indices.shape
    rows = np.repeat(np.arange(n), k)
    cols = knn_indices.ravel()
    diff = (dists - rhos[:, None].astype(np.float32)).astype(np.float32)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        ex = np.exp(-(diff / sigmas[:, None].astype(np.float32))).astype(np.float32)
    val = np.where((diff <= 0) | (sigmas[:, None] == 0), np.float32(1.0), ex).astype(np.float32)
    val = np.where(knn_indices == np.arange(n)[:, None], np.float32(0.0), val).ravel()
    m = sp.coo_matrix((val, (rows, cols)), shape=(n, n))
    m.eliminate_zeros()
    return m


def fuzzy_union(directed) -> sp.csr_matrix:
    """Stage 4: A + A^T - A∘A^T (f32 CSR, duplicates summed, zeros removed)."""
    a = sp.csr_matrix(directed)
    s = a + a.T - a.multiply(a.T)
    s = sp.csr_matrix(s)
    s.sum_duplicates()
    s.eliminate_zeros()
    return s


def prune(g, n: int) -> sp.csr_matrix:
    """Stage 5a: entries below max / n_epochs removed."""
    g = sp.csr_matrix(g).copy()
    n_epochs = 500 if n <= 10000 else 200
    thr = g.data.max() / float(n_epochs)
    g.data[g.data < thr] = 0.0
    g.eliminate_zeros()
    return g


def fuzzy_graph(x: np.ndarray, k: int) -> sp.csr_matrix:
    """All five stages from the points."""
    idx, d = knn_exact(x, k)
    sig, rho = smooth_knn(d, k)
    return prune(fuzzy_union(membership(idx, d, sig, rho)), x.shape[0])
