"""Synthetic UMAP fuzzy-kNN graphs built on the GPU (benchmark and test input).

This is input synthesis, not part of the eigensolve path: it uses torch
(cuBLAS GEMM distances + top-k) to build, at n = 10^6, the same graph the CPU
generator ``oracle.graphgen`` builds for small n:

1. exact kNN by brute force (||q||^2 + ||x||^2 - 2 q.x in f32, GEMM with
   TF32 disabled), each point its own first neighbour;
2. smooth-kNN calibration (rho = nearest non-self distance, sigma by 64-step
   bisection to sum exp(-(d - rho)/sigma) = log2 k, floor 1e-3 * mean d);
3. memberships exp(-(d - rho)/sigma), fuzzy union A + A^T - A o A^T in f32
   (the same operation order as scipy, so the result is bitwise symmetric);
4. prune below max/200 (n > 10000) or max/500.
"""
from __future__ import annotations

import math

import numpy as np


def _torch():
    import torch
    return torch


def gaussian_mixture_gpu(n: int, n_clusters: int, dims: int, seed: int = 42, center_std: float = 5.0,
                         background_frac: float = 0.0, anisotropic: bool = False,
                         dirichlet_alpha: float | None = None, device="cuda"):
    """Seeded Gaussian mixture (float32 [n, dims]) generated on the GPU."""
    torch = _torch()
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n_bg = int(round(n * background_frac))
    n_cl = n - n_bg
    centers = torch.randn(n_clusters, dims, generator=g, device=device, dtype=torch.float64) * center_std
    if dirichlet_alpha is None:
        sizes = np.full(n_clusters, n_cl // n_clusters)
        sizes[: n_cl - sizes.sum()] += 1
    else:
        rng = np.random.default_rng(seed)
        p = rng.dirichlet(np.full(n_clusters, dirichlet_alpha))
        sizes = np.floor(p * n_cl).astype(np.int64)
        sizes[np.argsort(-p)[: n_cl - sizes.sum()]] += 1
    parts = []
    for c in range(n_clusters):
        z = torch.randn(int(sizes[c]), dims, generator=g, device=device, dtype=torch.float64)
        if anisotropic:
            q, _ = torch.linalg.qr(torch.randn(dims, dims, generator=g, device=device, dtype=torch.float64))
            ev = torch.rand(dims, generator=g, device=device, dtype=torch.float64) * 1.8 + 0.2
            z = (z * ev.sqrt()) @ q.T
        parts.append(z + centers[c])
    x = torch.cat(parts, 0)
    if n_bg:
        lo = x.min(0).values
        hi = x.max(0).values
        u = torch.rand(n_bg, dims, generator=g, device=device, dtype=torch.float64)
        x = torch.cat([x, lo + u * (hi - lo)], 0)
    return x.float().contiguous()


def knn_gpu(x, k: int, chunk: int = 4096):
    """(indices int64 [n, k], distances f32 [n, k]); column 0 is the point itself."""
    torch = _torch()
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = x.shape[0]
        sq = (x * x).sum(1)
        idx = torch.empty(n, k, dtype=torch.int64, device=x.device)
        dist = torch.empty(n, k, dtype=torch.float32, device=x.device)
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            d = sq[s:e, None] + sq[None, :] - 2.0 * (x[s:e] @ x.T)
            rows = torch.arange(s, e, device=x.device)
            d[rows - s, rows] = -1.0  # self first
            v, i = torch.topk(d, k, dim=1, largest=False, sorted=True)
            v[:, 0] = 0.0
            idx[s:e] = i
            dist[s:e] = v.clamp_min(0.0).sqrt()
            del d
        return idx, dist
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def smooth_knn_gpu(dist, k: int, n_iter: int = 64):
    torch = _torch()
    d = dist.double()
    target = math.log2(k)
    nz = torch.where(d > 0, d, torch.full_like(d, float("inf")))
    rho = nz.min(1).values
    rho = torch.where(torch.isinf(rho), torch.zeros_like(rho), rho)
    diff = d[:, 1:] - rho[:, None]
    n = d.shape[0]
    lo = torch.zeros(n, dtype=torch.float64, device=d.device)
    hi = torch.full((n,), float("inf"), dtype=torch.float64, device=d.device)
    mid = torch.ones(n, dtype=torch.float64, device=d.device)
    done = torch.zeros(n, dtype=torch.bool, device=d.device)
    for _ in range(n_iter):
        terms = torch.where(diff > 0, torch.exp(-diff.clamp_min(0) / mid[:, None]), torch.ones_like(diff))
        psum = terms.sum(1)
        done |= (psum - target).abs() < 1e-5
        act = ~done
        gt = act & (psum > target)
        hi = torch.where(gt, mid, hi)
        mid = torch.where(gt, (lo + hi) / 2, mid)
        le = act & ~(psum > target)
        lo = torch.where(le, mid, lo)
        mid = torch.where(le & torch.isinf(hi), mid * 2, torch.where(le, (lo + hi) / 2, mid))
    floor = torch.where(rho > 0, 1e-3 * d.mean(1), 1e-3 * d.mean())
    sigma = torch.where(mid < floor, floor, mid)
    return sigma.float(), rho.float()


def fuzzy_graph_gpu(idx, dist, sigma, rho, prune: bool = True):
    """Symmetric fuzzy union as CSR (indptr int64, indices int32, data f32) on the GPU."""
    torch = _torch()
    n, k = idx.shape
    dev = idx.device
    diff = dist - rho[:, None]
    val = torch.where((diff <= 0) | (sigma[:, None] == 0), torch.ones_like(dist), torch.exp(-diff / sigma[:, None]))
    rows = torch.arange(n, device=dev).repeat_interleave(k)
    cols = idx.reshape(-1)
    v = val.reshape(-1)
    keep = (cols != rows) & (v != 0)
    rows, cols, v = rows[keep], cols[keep], v[keep]
    fkey = rows * n + cols
    order = torch.argsort(fkey)
    fkey, v = fkey[order], v[order]
    rkey = cols[order] * n + rows[order]
    ukey = torch.unique(torch.cat([fkey, rkey]))

    def lookup(keys):
        pos = torch.searchsorted(fkey, keys).clamp_max(fkey.numel() - 1)
        hit = fkey[pos] == keys
        return torch.where(hit, v[pos], torch.zeros_like(v[pos]))

    a = lookup(ukey)
    b = lookup((ukey % n) * n + ukey // n)
    w = (a + b) - (a * b)
    keep = w != 0
    if prune:
        thr = w.max() / (500.0 if n <= 10000 else 200.0)
        keep &= ~(w < thr)
    ukey, w = ukey[keep], w[keep]
    r = ukey // n
    c = (ukey % n).to(torch.int32)
    counts = torch.bincount(r, minlength=n)
    indptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    indptr[1:] = torch.cumsum(counts, 0)
    return indptr, c.contiguous(), w.contiguous()


def fuzzy_knn_graph_gpu(n: int, k: int = 15, n_clusters: int = 100, dims: int = 50, seed: int = 42,
                        center_std: float = 5.0, background_frac: float = 0.05, anisotropic: bool = False,
                        dirichlet_alpha: float | None = None, device="cuda"):
    x = gaussian_mixture_gpu(n, n_clusters, dims, seed, center_std, background_frac, anisotropic,
                             dirichlet_alpha, device)
    idx, dist = knn_gpu(x, k)
    sigma, rho = smooth_knn_gpu(dist, k)
    return fuzzy_graph_gpu(idx, dist, sigma, rho)


def multi_component_graph_gpu(n_comp: int = 500, size_min: int = 20, size_max: int = 100_000, dims: int = 20,
                              k: int = 15, seed: int = 42, device="cuda"):
    """Block-diagonal union of independent fuzzy-kNN graphs (the batched
    multi-component workload): component sizes log-uniform in [size_min,
    size_max], each a seeded Gaussian mixture of 1-10 overlapping clusters in
    `dims` dimensions, shifted to its own region of the data space.  Returns
    (indptr int64, indices int32, data f32, n, points f32 [n, dims], sizes)."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(size_min), math.log(size_max), n_comp)).astype(np.int64)
    ips, ixs, dvs, xs = [], [], [], []
    node_off = 0
    nnz_off = 0
    for c, sz in enumerate(sizes):
        sz = int(sz)
        kk = min(k, sz - 1)
        clusters = int(rng.integers(1, 11))
        x = gaussian_mixture_gpu(sz, clusters, dims, seed * 100_003 + c, center_std=1.0, device=device)
        x = x + torch.from_numpy(rng.normal(0.0, 100.0, dims).astype(np.float32)).to(x.device)
        idx, dist = knn_gpu(x, kk)
        sigma, rho = smooth_knn_gpu(dist, kk)
        ip, ix, dv = fuzzy_graph_gpu(idx, dist, sigma, rho, prune=False)
        ips.append(ip[:-1] + nnz_off)
        ixs.append(ix + node_off)
        dvs.append(dv)
        xs.append(x)
        node_off += sz
        nnz_off += int(ix.numel())
    indptr = torch.cat(ips + [torch.tensor([nnz_off], dtype=torch.int64, device=device)])
    return indptr, torch.cat(ixs).contiguous(), torch.cat(dvs).contiguous(), node_off, torch.cat(xs), sizes


def to_scipy(indptr, indices, data, n):
    import scipy.sparse as sp
    return sp.csr_matrix((data.cpu().numpy(), indices.cpu().numpy(), indptr.cpu().numpy()), shape=(n, n))
