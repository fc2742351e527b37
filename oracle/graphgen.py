"""Seeded synthetic UMAP fuzzy-kNN graphs (CPU; test and benchmark input).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.

The construction restates the fuzzy simplicial set of McInnes, Healy and
Melville (UMAP, arXiv:1802.03426, sec. 3 and its smooth-kNN calibration),
which is the graph the spectral-init crate receives from umap-rs:

1. exact k nearest neighbours, each point its own first neighbour (d = 0);
2. rho_i = distance to the nearest non-identical neighbour; sigma_i by
   bisection (64 steps, tolerance 1e-5) so that
   sum_{j>=1} exp(-max(0, d_ij - rho_i) / sigma_i) = log2(k), with the
   floor sigma_i >= 1e-3 * mean_j d_ij;
3. directed weights w_ij = exp(-max(0, d_ij - rho_i) / sigma_i) (0 for self);
4. fuzzy union W = A + A^T - A o A^T;
5. prune entries below max(W) / n_epochs (500 epochs for n <= 10000, else 200).

The generators of the benchmark workloads (Gaussian mixtures with optional
anisotropic covariances, Dirichlet cluster sizes and a uniform background)
follow the workload descriptions of the spectral-init performance plan; every
free parameter is an argument with a recorded default.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

SMOOTH_K_TOLERANCE = 1e-5
MIN_K_DIST_SCALE = 1e-3


def gaussian_mixture(n: int, n_clusters: int, dims: int, seed: int = 42, center_std: float = 5.0,
                     anisotropic: bool = False, dirichlet_alpha: float | None = None,
                     background_frac: float = 0.0, cluster_std: float = 1.0) -> np.ndarray:
    """Points of a seeded Gaussian mixture (float32, cluster by cluster).

    centers ~ N(0, center_std^2 I); isotropic clusters have std ``cluster_std``;
    anisotropic clusters get a random rotation and axis variances U[0.2, 2];
    cluster sizes are equal or ~ Dirichlet(alpha); ``background_frac`` of the
    points are uniform over the bounding box of the clustered points.
    """
    rng = np.random.default_rng(seed)
    n_bg = int(round(n * background_frac))
    n_cl = n - n_bg
    centers = rng.normal(0.0, center_std, size=(n_clusters, dims))
    if dirichlet_alpha is None:
        sizes = np.full(n_clusters, n_cl // n_clusters)
        sizes[: n_cl - sizes.sum()] += 1
    else:
        p = rng.dirichlet(np.full(n_clusters, dirichlet_alpha))
        sizes = np.floor(p * n_cl).astype(np.int64)
        sizes[np.argsort(-p)[: n_cl - sizes.sum()]] += 1
    parts = []
    for c in range(n_clusters):
        z = rng.standard_normal((int(sizes[c]), dims))
        if anisotropic:
            q, _ = np.linalg.qr(rng.standard_normal((dims, dims)))
            ev = rng.uniform(0.2, 2.0, size=dims)
            z = (z * np.sqrt(ev)) @ q.T
        else:
            z = z * cluster_std
        parts.append(z + centers[c])
    x = np.concatenate(parts, axis=0) if parts else np.zeros((0, dims))
    if n_bg:
        lo, hi = x.min(axis=0), x.max(axis=0)
        x = np.concatenate([x, rng.uniform(lo, hi, size=(n_bg, dims))], axis=0)
    return x.astype(np.float32)


def exact_knn(x: np.ndarray, k: int):
    """(indices int64 [n, k], distances float32 [n, k]); column 0 is the point itself."""
    from sklearn.neighbors import NearestNeighbors

    nn = NearestNeighbors(n_neighbors=k, algorithm="auto")
    nn.fit(x.astype(np.float64))
    d, i = nn.kneighbors(x.astype(np.float64))
    # make the point itself the first neighbour even with duplicate points
    for r in np.nonzero(i[:, 0] != np.arange(len(x)))[0]:
        row = list(i[r])
        if r in row:
            j = row.index(r)
            i[r, [0, j]] = i[r, [j, 0]]
            d[r, [0, j]] = d[r, [j, 0]]
        else:
            i[r, 1:] = i[r, :-1]
            d[r, 1:] = d[r, :-1]
            i[r, 0] = r
            d[r, 0] = 0.0
    return i.astype(np.int64), d.astype(np.float32)


def smooth_knn_dist(dists: np.ndarray, k: float, n_iter: int = 64, local_connectivity: float = 1.0,
                    bandwidth: float = 1.0):
    """Vectorised bisection for sigma_i and rho_i (float32 inputs, float64 work)."""
    d = dists.astype(np.float64)
    n = d.shape[0]
    target = math.log2(k) * bandwidth
    rho = np.zeros(n)
    for i in range(n):
        nz = d[i][d[i] > 0.0]
        if nz.shape[0] >= local_connectivity:
            idx = int(math.floor(local_connectivity))
            interp = local_connectivity - idx
            if idx > 0:
                rho[i] = nz[idx - 1]
                if interp > SMOOTH_K_TOLERANCE:
                    rho[i] += interp * (nz[idx] - nz[idx - 1])
            else:
                rho[i] = interp * nz[0]
        elif nz.shape[0] > 0:
            rho[i] = nz.max()
    lo = np.zeros(n)
    hi = np.full(n, np.inf)
    mid = np.ones(n)
    done = np.zeros(n, dtype=bool)
    diff = d[:, 1:] - rho[:, None]
    for _ in range(n_iter):
        terms = np.where(diff > 0.0, np.exp(-np.maximum(diff, 0.0) / mid[:, None]), 1.0)
        psum = terms.sum(axis=1)
        newly = (~done) & (np.abs(psum - target) < SMOOTH_K_TOLERANCE)
        done |= newly
        act = ~done
        gt = act & (psum > target)
        hi = np.where(gt, mid, hi)
        mid = np.where(gt, (lo + hi) / 2.0, mid)
        le = act & ~(psum > target)
        lo = np.where(le, mid, lo)
        mid = np.where(le & np.isinf(hi), mid * 2.0, np.where(le, (lo + hi) / 2.0, mid))
        if done.all():
            break
    sigma = mid
    mean_all = d.mean()
    mean_i = d.mean(axis=1)
    floor = np.where(rho > 0.0, MIN_K_DIST_SCALE * mean_i, MIN_K_DIST_SCALE * mean_all)
    sigma = np.where(sigma < floor, floor, sigma)
    return sigma.astype(np.float32), rho.astype(np.float32)


def membership_strengths(knn_i: np.ndarray, knn_d: np.ndarray, sigma: np.ndarray, rho: np.ndarray, n: int):
    d = knn_d.astype(np.float32)
    diff = d - rho[:, None]
    safe_sigma = np.where(sigma == 0.0, np.float32(1.0), sigma)[:, None]
    val = np.where((diff <= 0.0) | (sigma[:, None] == 0.0), np.float32(1.0),
                   np.exp(-np.maximum(diff, 0.0) / safe_sigma)).astype(np.float32)
    rows = np.repeat(np.arange(n), knn_i.shape[1])
    cols = knn_i.reshape(-1)
    v = val.reshape(-1)
    v[cols == rows] = 0.0
    a = sp.coo_matrix((v, (rows, cols)), shape=(n, n)).tocsr()
    a.eliminate_zeros()
    return a


def fuzzy_union(a: sp.csr_matrix) -> sp.csr_matrix:
    at = a.T.tocsr()
    s = (a + at - a.multiply(at)).tocsr()
    s.sum_duplicates()
    s.eliminate_zeros()
    return s


def prune(s: sp.csr_matrix, n_epochs: int | None = None) -> sp.csr_matrix:
    n = s.shape[0]
    if n_epochs is None:
        n_epochs = 500 if n <= 10000 else 200
    g = s.copy()
    if g.nnz:
        thr = g.data.max() / float(n_epochs)
        g.data[g.data < thr] = 0.0
        g.eliminate_zeros()
    return g


def fuzzy_knn_graph(x: np.ndarray, k: int, do_prune: bool = True) -> sp.csr_matrix:
    """The f32 fuzzy-kNN graph (sorted CSR) of points ``x``."""
    n = x.shape[0]
    ki, kd = exact_knn(x, k)
    sigma, rho = smooth_knn_dist(kd, float(k))
    a = membership_strengths(ki, kd, sigma, rho, n)
    g = fuzzy_union(a)
    if do_prune:
        g = prune(g)
    g = sp.csr_matrix(g, dtype=np.float32)
    g.sort_indices()
    return g


def degrees_f64(g: sp.csr_matrix):
    deg = np.asarray(g.astype(np.float64).sum(axis=1)).ravel()
    return deg, np.sqrt(deg)


def path_graph(n: int) -> sp.csr_matrix:
    r = np.concatenate([np.arange(n - 1), np.arange(1, n)])
    c = np.concatenate([np.arange(1, n), np.arange(n - 1)])
    g = sp.csr_matrix((np.ones(len(r), np.float32), (r, c)), shape=(n, n))
    g.sort_indices()
    return g


def ring_graph(n: int, half: int = 2) -> sp.csr_matrix:
    rows, cols = [], []
    for o in range(1, half + 1):
        i = np.arange(n)
        rows += [i, i]
        cols += [(i + o) % n, (i - o) % n]
    g = sp.csr_matrix((np.ones(sum(len(r) for r in rows), np.float32), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    g.sum_duplicates()
    g.data[:] = 1.0
    g.sort_indices()
    return g


def block_diagonal(graphs) -> sp.csr_matrix:
    g = sp.block_diag(graphs, format="csr", dtype=np.float32)
    g.sort_indices()
    return g
