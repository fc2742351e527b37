"""numpy/scipy restatement of the spectral-init eigensolve path (CPU oracle).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Every function names the
reference file and lines it restates (paths inside the spectral-init crate).

Data conventions
----------------
* A graph is a scipy ``csr_matrix`` with ``float32`` weights (the crate's
  ``CsMatI<f32, u32, usize>``) and sorted column indices.
* Blocks of vectors are ``float64`` arrays of shape ``[n, k]`` (row-major, like
  the crate's ``Array2<f64>``).
* Random numbers come from ``numpy.random.default_rng(seed)``.  The crate uses
  ``StdRng`` (ChaCha12) + ``rand_distr``; those streams are not reproducible
  outside Rust, so parity is stated on eigenvalues, residuals and subspaces,
  never on the random bits.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# --------------------------------------------------------------------------
# Constants (src/metrics.rs:20-52, src/solvers/lobpcg.rs:60-97,
# src/solvers/mod.rs:32, src/solvers/sinv.rs:18)
# --------------------------------------------------------------------------
RSVD_QUALITY_THRESHOLD = 1e-2
DENSE_EVD_QUALITY_THRESHOLD = 1e-6
LOBPCG_QUALITY_THRESHOLD = 1e-5
SINV_LOBPCG_QUALITY_THRESHOLD = 1e-6
LOBPCG_ACCEPT_TOL = 1e-5
SINV_LINFA_TOL = 1e-8
DEGENERATE_GAP_THRESHOLD = 1e-6
SUBSPACE_GRAM_DET_THRESHOLD = 0.95

REGULARIZATION_EPS = 1e-5
CHEB_LOWER_BOUND = 0.1
CHEB_UPPER_BOUND = 2.0
CHEB_DEGREE = 8
CHEB_MIN_N = 1000
MAX_WARM_RESTARTS = 3
LOBPCG_INITIAL_MAXITER_CAP = 300
LOBPCG_RESTART_MAXITER_CAP = 1000
DENSE_N_THRESHOLD = 2000
SINV_SHIFT = 1e-4

PYTHON_COMPAT = 0
RUST_NATIVE = 1


class SpectralError(Exception):
    """Mirror of ``SpectralError`` (src/lib.rs:167-182)."""


class ConvergenceFailure(SpectralError):
    pass


class InvalidGraph(SpectralError):
    pass


class TooFewNodes(SpectralError):
    def __init__(self, n, dims):
        super().__init__(f"graph has too few nodes ({n}) for {dims}-dimensional embedding")
        self.n = n
        self.dims = dims


def f32_tol(x: float) -> float:
    """The crate passes ``tol`` to linfa as ``f32`` (src/solvers/lobpcg.rs:307)."""
    return float(np.float32(x))


# --------------------------------------------------------------------------
# L1: degrees and Laplacian (src/laplacian.rs:8-88)
# --------------------------------------------------------------------------
def column_sum_f32(graph: sp.csr_matrix) -> np.ndarray:
    """f32 column scatter ``deg[col] += val`` in CSR iteration order
    (src/laplacian.rs:8-16).  ``np.add.at`` applies the additions one element at
    a time in index order with a float32 accumulator, which is exactly the
    crate's loop."""
    n = graph.shape[1]
    deg = np.zeros(n, dtype=np.float32)
    np.add.at(deg, graph.indices.astype(np.int64), graph.data.astype(np.float32))
    return deg


def compute_degrees(graph: sp.csr_matrix, mode: int = PYTHON_COMPAT):
    """src/laplacian.rs:29-49.  PythonCompat: f32 column scatter widened to f64.
    RustNative: per-row sequential f64 sum of the f32 weights."""
    n = graph.shape[0]
    if mode == PYTHON_COMPAT:
        degrees = column_sum_f32(graph).astype(np.float64)
    else:
        degrees = np.zeros(n, dtype=np.float64)
        ip = graph.indptr
        d = graph.data.astype(np.float64)
        for i in range(n):
            s = 0.0
            for v in d[ip[i]:ip[i + 1]]:
                s += v
            degrees[i] = s
    return degrees, np.sqrt(degrees)


def compute_degrees_rust_native_fast(graph: sp.csr_matrix):
    """Vectorised RustNative degrees for large graphs: ``np.add.reduceat`` sums
    each row left to right in f64 (same order as the sequential loop for rows
    with at least one entry)."""
    n = graph.shape[0]
    d = graph.data.astype(np.float64)
    ip = graph.indptr.astype(np.int64)
    out = np.zeros(n)
    nz = ip[1:] > ip[:-1]
    if d.size:
        sums = np.add.reduceat(d, ip[:-1][nz])
        out[nz] = sums
    return out, np.sqrt(out)


def inv_sqrt(sqrt_deg: np.ndarray) -> np.ndarray:
    """``if s > 0 { 1/s } else { 0 }`` (src/lib.rs:233-236)."""
    out = np.zeros_like(sqrt_deg)
    pos = sqrt_deg > 0.0
    out[pos] = 1.0 / sqrt_deg[pos]
    return out


def build_normalized_laplacian(graph: sp.csr_matrix, inv_sqrt_deg: np.ndarray) -> sp.csr_matrix:
    """src/laplacian.rs:60-88: off-diagonal ``-inv[i] * w_ij * inv[j]`` (evaluated
    left to right in f64), self loops skipped, unit diagonal for every node,
    CSR with sorted columns and duplicates summed (``TriMat::to_csr``)."""
    n = graph.shape[0]
    coo = graph.tocoo()
    r = coo.row.astype(np.int64)
    c = coo.col.astype(np.int64)
    w = coo.data.astype(np.float64)
    off = r != c
    r, c, w = r[off], c[off], w[off]
    vals = (-inv_sqrt_deg[r]) * w * inv_sqrt_deg[c]
    rows = np.concatenate([r, np.arange(n)])
    cols = np.concatenate([c, np.arange(n)])
    data = np.concatenate([vals, np.ones(n)])
    lap = sp.csr_matrix((data, (rows, cols)), shape=(n, n))
    lap.sum_duplicates()
    lap.sort_indices()
    return lap


# --------------------------------------------------------------------------
# Components (src/components.rs:7-44)
# --------------------------------------------------------------------------
def find_components(graph: sp.csr_matrix):
    """BFS labelling in start-node order; labels are numbered by the smallest
    node of each component."""
    from collections import deque

    n = graph.shape[0]
    labels = np.full(n, -1, dtype=np.int64)
    ip, ix = graph.indptr, graph.indices
    nc = 0
    for start in range(n):
        if labels[start] != -1:
            continue
        labels[start] = nc
        q = deque([start])
        while q:
            node = q.popleft()
            for nb in ix[ip[node]:ip[node + 1]]:
                if labels[nb] == -1:
                    labels[nb] = nc
                    q.append(nb)
        nc += 1
    return labels, nc


def find_components_fast(graph: sp.csr_matrix):
    """Same partition and numbering as :func:`find_components` for symmetric
    graphs, via scipy (used for large n)."""
    from scipy.sparse.csgraph import connected_components

    nc, lab = connected_components(graph, directed=False)
    # renumber by smallest member node (BFS start order)
    n = graph.shape[0]
    first = np.full(nc, n, dtype=np.int64)
    np.minimum.at(first, lab, np.arange(n))
    order = np.argsort(first, kind="stable")
    remap = np.empty(nc, dtype=np.int64)
    remap[order] = np.arange(nc)
    return remap[lab].astype(np.int64), int(nc)


# --------------------------------------------------------------------------
# L2: operator (src/operator.rs:174-228)
# --------------------------------------------------------------------------
class CsrOperator:
    """``LinearOperator`` over an explicit CSR Laplacian: ``y = L x``."""

    def __init__(self, lap: sp.csr_matrix, shift: float = 0.0):
        self.lap = lap
        self.shift = shift
        self.n = lap.shape[0]
        self.applies = 0

    def apply(self, x: np.ndarray) -> np.ndarray:
        self.applies += 1
        y = self.lap @ x
        if self.shift:
            y = y + self.shift * x
        return np.asarray(y)

    def size(self):
        return self.n


# --------------------------------------------------------------------------
# Chebyshev filter (src/solvers/lobpcg.rs:113-150, :270-291)
# --------------------------------------------------------------------------
def chebyshev_precond(apply, r: np.ndarray, a: float, b: float, degree: int) -> np.ndarray:
    c = (a + b) / 2.0
    e = (b - a) / 2.0
    scale = 2.0 / e
    shift = scale * c
    y_prev = r.copy()
    ly = apply(r)
    y = (ly - c * r) / e
    for _ in range(2, degree + 1):
        ly = apply(y)
        y_new = scale * ly
        y_new -= shift * y
        y_new -= y_prev
        y_prev, y = y, y_new
    return y


def chebyshev_filter_start(apply, x0: np.ndarray) -> np.ndarray:
    """``X <- colnormalize((X + T_8 X) / 2)`` (src/solvers/lobpcg.rs:270-291)."""
    t = chebyshev_precond(apply, x0, CHEB_LOWER_BOUND, CHEB_UPPER_BOUND, CHEB_DEGREE)
    filt = (x0 + t) / 2.0
    out = np.zeros_like(filt)
    for j in range(filt.shape[1]):
        col = filt[:, j]
        nrm = math.sqrt(float(col @ col))
        out[:, j] = col / nrm if nrm > 1e-300 else col
    return out


# --------------------------------------------------------------------------
# LOBPCG core (restatement of linfa-linalg 0.2 ``lobpcg``; called at
# src/solvers/lobpcg.rs:327-358 and src/solvers/sinv.rs:139-153).
# Algorithm: Knyazev 2001 block LOBPCG with soft locking, residuals
# orthogonalised against X, Cholesky orthonormalisation, explicit Gram
# matrices, fallback to span{X,R} when span{X,R,P} is not numerically
# independent, and "best iterate" tracking by the sum of residual norms.
# --------------------------------------------------------------------------
class _NotPD(Exception):
    pass


@dataclass
class LobpcgResult:
    eigvals: np.ndarray
    eigvecs: np.ndarray
    rnorm: np.ndarray
    converged: bool
    iterations: int


def _ortho(v: np.ndarray):
    g = v.T @ v
    g = (g + g.T) / 2
    try:
        l = np.linalg.cholesky(g)
    except np.linalg.LinAlgError as e:  # not positive definite
        raise _NotPD() from e
    q = sla.solve_triangular(l, v.T, lower=True).T
    return q, l


def _sorted_eig(a, b, size, largest):
    try:
        if b is None:
            w, v = np.linalg.eigh(a)
        else:
            w, v = sla.eigh(a, b)
    except (np.linalg.LinAlgError, sla.LinAlgError) as e:
        raise _NotPD() from e
    if largest:
        idx = np.argsort(-w, kind="stable")[:size]
    else:
        idx = np.argsort(w, kind="stable")[:size]
    return w[idx], v[:, idx]


def lobpcg_core(apply, x: np.ndarray, tol: float, maxiter: int, largest: bool = False,
                callback=None) -> LobpcgResult:
    """``callback(iteration, residual_norms)`` may return True to stop early
    (treated like reaching ``maxiter``)."""
    n, size_x = x.shape
    try:
        x, _ = _ortho(x)
    except _NotPD:
        return LobpcgResult(None, None, None, False, 0)
    ax = apply(x)
    xax = x.T @ ax
    lam, blk = _sorted_eig((xax + xax.T) / 2, None, size_x, largest)
    x = x @ blk
    ax = ax @ blk
    active = np.ones(size_x, dtype=bool)
    best = None
    p = ap = None
    it = 0
    converged = False
    while True:
        r = ax - x * lam[None, :]
        rn = np.sqrt(np.sum(r * r, axis=0))
        s = float(np.sum(rn))
        if best is None or best[3] > s:
            best = (lam.copy(), x.copy(), rn.copy(), s)
        active = active & (rn > tol)
        m = int(active.sum())
        if m == 0:
            converged = True
            break
        if it >= maxiter:
            break
        if callback is not None and callback(it, rn):
            break
        it += 1
        ra = r[:, active]
        ra = ra - x @ (x.T @ ra)
        try:
            ra, _ = _ortho(ra)
        except _NotPD:
            break
        ar = apply(ra)
        xar = x.T @ ar
        rar = ra.T @ ar
        rar = (rar + rar.T) / 2
        xax = x.T @ ax
        xax = (xax + xax.T) / 2
        xx = x.T @ x
        rr = ra.T @ ra
        xr = x.T @ ra
        pa = apa = None
        if p is not None:
            try:
                pa, pr = _ortho(p[:, active])
                apa = sla.solve_triangular(pr, ap[:, active].T, lower=True).T
            except _NotPD:
                pa = apa = None
        res = None
        if pa is not None:
            xap = x.T @ apa
            rap = ra.T @ apa
            pap = pa.T @ apa
            pap = (pap + pap.T) / 2
            xp = x.T @ pa
            rp = ra.T @ pa
            pp = pa.T @ pa
            ga = np.block([[xax, xar, xap], [xar.T, rar, rap], [xap.T, rap.T, pap]])
            gb = np.block([[xx, xr, xp], [xr.T, rr, rp], [xp.T, rp.T, pp]])
            try:
                res = _sorted_eig(ga, gb, size_x, largest)
            except _NotPD:
                res = None
        if res is None:
            pa = apa = None
            ga = np.block([[xax, xar], [xar.T, rar]])
            gb = np.block([[xx, xr], [xr.T, rr]])
            try:
                res = _sorted_eig(ga, gb, size_x, largest)
            except _NotPD:
                break
        lam, ev = res
        tau = ev[:size_x]
        alpha = ev[size_x:size_x + m]
        if pa is not None:
            gamma = ev[size_x + m:]
            pn = ra @ alpha + pa @ gamma
            apn = ar @ alpha + apa @ gamma
        else:
            pn = ra @ alpha
            apn = ar @ alpha
        x = x @ tau + pn
        ax = ax @ tau + apn
        p, ap = pn, apn
    lam_b, x_b, rn_b, _ = best
    return LobpcgResult(lam_b, x_b, rn_b, converged, it)


# --------------------------------------------------------------------------
# Rayleigh-Ritz refine + residuals (src/solvers/lobpcg.rs:158-223)
# --------------------------------------------------------------------------
def rayleigh_ritz_refine(apply, vecs: np.ndarray):
    ax = apply(vecs)
    g = vecs.T @ ax
    try:
        w, v = np.linalg.eigh(g)  # lower triangle, like faer Side::Lower
    except np.linalg.LinAlgError:
        return None
    return w, vecs @ v


def per_vector_residuals(apply, vals: np.ndarray, vecs: np.ndarray) -> np.ndarray:
    ax = apply(vecs)
    out = np.empty(len(vals))
    for i, lam in enumerate(vals):
        v = vecs[:, i]
        cn = max(math.sqrt(float(v @ v)), np.finfo(np.float64).eps)
        d = ax[:, i] - lam * v
        out[i] = math.sqrt(float(d @ d)) / cn
    return out


def initial_block(n: int, k: int, seed: int, sqrt_deg: np.ndarray) -> np.ndarray:
    """Random ``N(0,1)`` block with the trivial-vector hint in column 0
    (src/solvers/lobpcg.rs:243-252)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, k))
    nrm = math.sqrt(float(sqrt_deg @ sqrt_deg))
    if nrm > 0.0:
        x[:, 0] = sqrt_deg / nrm
    return x


def lobpcg_solve(op, n_components: int, seed: int, regularize: bool, sqrt_deg: np.ndarray,
                 x_init: np.ndarray | None = None, stats: dict | None = None):
    """src/solvers/lobpcg.rs:227-465.  Returns ``((vals, vecs), restart_count)``
    or ``None``.  ``x_init`` replaces the seeded random start (used to feed a
    warm-start block); the Chebyshev filter is still applied for n >= 1000."""
    n = op.size()
    k = n_components + 1
    if n_components == 0 or k >= n or len(sqrt_deg) != n:
        return None
    x0 = initial_block(n, k, seed, sqrt_deg) if x_init is None else np.array(x_init, dtype=np.float64)

    def l_apply(x):
        return op.apply(x)

    if n >= CHEB_MIN_N:
        x0 = chebyshev_filter_start(l_apply, x0)

    if regularize:
        def a_apply(x):
            return op.apply(x) + REGULARIZATION_EPS * x
    else:
        a_apply = l_apply

    tol = f32_tol(LOBPCG_ACCEPT_TOL)
    last = None
    restart_count = 0
    x_init_cur = x0
    total_iters = 0
    for restart in range(MAX_WARM_RESTARTS + 1):
        cap = LOBPCG_INITIAL_MAXITER_CAP if restart == 0 else LOBPCG_RESTART_MAXITER_CAP
        maxiter = min(n * 5, cap)
        res = lobpcg_core(a_apply, x_init_cur, tol, maxiter)
        total_iters += res.iterations
        if res.eigvals is None:
            break
        if res.converged or np.all(res.rnorm < LOBPCG_ACCEPT_TOL):
            raw = (res.eigvals, res.eigvecs)
        else:
            if restart < MAX_WARM_RESTARTS:
                x_init_cur = res.eigvecs
                continue
            break
        refined = rayleigh_ritz_refine(l_apply, raw[1])
        if refined is None:
            if restart < MAX_WARM_RESTARTS:
                x_init_cur = raw[1]
                continue
            break
        resid = per_vector_residuals(l_apply, refined[0], refined[1])
        if np.all(resid < LOBPCG_ACCEPT_TOL):
            if stats is not None:
                stats.update(iterations=total_iters, restarts=restart_count)
            return refined, restart_count
        restart_count += 1
        if restart < MAX_WARM_RESTARTS:
            x_init_cur = refined[1].copy()
        last = refined
    if stats is not None:
        stats.update(iterations=total_iters, restarts=restart_count)
    if last is None:
        return None
    return last, restart_count


# --------------------------------------------------------------------------
# Shift-invert LOBPCG (src/solvers/sinv.rs:106-189)
# --------------------------------------------------------------------------
def lobpcg_sinv_solve(lap: sp.csr_matrix, n_components: int, seed: int, sqrt_deg: np.ndarray):
    n = lap.shape[0]
    k = n_components + 1
    if n_components == 0 or k >= n or len(sqrt_deg) != n:
        return None
    m = (lap + SINV_SHIFT * sp.identity(n, format="csr")).tocsc()
    try:
        solve = spla.factorized(m)
    except RuntimeError:
        return None

    def apply(x):
        return np.column_stack([solve(x[:, j].copy()) for j in range(x.shape[1])])

    x0 = initial_block(n, k, seed, sqrt_deg)
    res = lobpcg_core(apply, x0, f32_tol(SINV_LINFA_TOL), min(n * 5, 300), largest=True)
    if res.eigvals is None:
        return None
    if not (res.converged or np.all(res.rnorm < SINV_LOBPCG_QUALITY_THRESHOLD)):
        return None
    vals = 1.0 / res.eigvals - SINV_SHIFT
    order = np.argsort(vals, kind="stable")
    return vals[order], res.eigvecs[:, order]


# --------------------------------------------------------------------------
# Randomized SVD via 2I - L (src/solvers/rsvd.rs:16-213)
# --------------------------------------------------------------------------
def two_i_minus_laplacian(lap: sp.csr_matrix) -> sp.csr_matrix:
    m = lap.copy().tocoo()
    diag = m.row == m.col
    data = -m.data
    data[diag] = 2.0 - m.data[diag]
    out = sp.csr_matrix((data, (m.row, m.col)), shape=lap.shape)
    out.sum_duplicates()
    out.sort_indices()
    return out


def rsvd_k_sub(n: int, rank: int) -> int:
    over = min(max(n // 10, max(rank, 5)), max(n - rank, 0))
    return min(rank + over, n)


def rsvd_solve(lap: sp.csr_matrix, n_components: int, seed: int, oversampling: int | None = None,
               nbiter: int = 2):
    n = lap.shape[0]
    assert 0 < n_components < n
    rank = n_components + 1
    k = rsvd_k_sub(n, rank) if oversampling is None else min(rank + oversampling, n)
    m = two_i_minus_laplacian(lap)
    rng = np.random.default_rng(seed)
    omega = rng.standard_normal((n, k))
    for _ in range(nbiter):
        omega = np.linalg.qr(m @ omega)[0]
        omega = np.linalg.qr(m @ omega)[0]
    q = np.linalg.qr(m @ omega)[0]
    b = q.T @ (m @ q)
    w, ub = np.linalg.eigh(b)
    v = q @ ub
    an = len(w)
    idx = [an - 1] + [max(an - 2 - i, 0) for i in range(n_components)]
    vals = np.array([2.0 - w[i] for i in idx])
    return vals, v[:, idx]


# --------------------------------------------------------------------------
# Dense EVD (src/solvers/dense.rs:9-46)
# --------------------------------------------------------------------------
def dense_evd(lap: sp.csr_matrix, k: int):
    n = lap.shape[0]
    if k > n:
        raise TooFewNodes(n, k)
    w, v = np.linalg.eigh(lap.toarray())
    return w[:k].copy(), v[:, :k].copy()


# --------------------------------------------------------------------------
# Quality gates (src/metrics.rs:57-92)
# --------------------------------------------------------------------------
def eigenpair_residual(lap: sp.csr_matrix, v: np.ndarray, lam: float) -> float:
    lv = lap @ v
    d = lv - lam * v
    return math.sqrt(float(d @ d)) / max(math.sqrt(float(v @ v)), 1e-300)


def max_eigenpair_residual(lap, vals, vecs) -> float:
    acc = 0.0
    for i, lam in enumerate(vals):
        r = eigenpair_residual(lap, vecs[:, i], lam)
        if math.isnan(acc) or math.isnan(r):
            acc = float("nan")
        else:
            acc = max(acc, r)
    return acc


def subspace_gram_det_kd(computed: np.ndarray, reference: np.ndarray) -> float:
    """src/metrics.rs:247-288: |det| of the column-normalised cross Gram."""
    def nrm(m):
        return m / np.maximum(np.linalg.norm(m, axis=0), np.finfo(np.float64).eps)

    g = nrm(reference).T @ nrm(computed)
    w = np.linalg.eigvalsh(g.T @ g)
    return float(math.sqrt(float(np.prod(np.maximum(w, 0.0)))))


def principal_angles(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Principal angles (radians) between span(a) and span(b)."""
    qa = np.linalg.qr(a)[0]
    qb = np.linalg.qr(b)[0]
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    return np.arccos(np.clip(s, -1.0, 1.0))


def sin_theta_max(a: np.ndarray, b: np.ndarray) -> float:
    """Largest principal-angle sine between span(a) and span(b), computed as
    ``||(I - Qb Qb^T) Qa||_2`` (accurate for tiny angles, unlike arccos)."""
    qa = np.linalg.qr(a)[0]
    qb = np.linalg.qr(b)[0]
    r = qa - qb @ (qb.T @ qa)
    return float(np.linalg.norm(r, 2))


# --------------------------------------------------------------------------
# Solver escalation chain (src/solvers/mod.rs:70-224)
# --------------------------------------------------------------------------
def solve_eigenproblem(lap: sp.csr_matrix, n_components: int, seed: int, sqrt_deg: np.ndarray,
                       dense_threshold: int = DENSE_N_THRESHOLD, skip_levels=(), stats: dict | None = None):
    n = lap.shape[0]
    op = CsrOperator(lap)
    if n < dense_threshold and 0 not in skip_levels:
        try:
            vals, vecs = dense_evd(lap, n_components + 1)
            if max_eigenpair_residual(lap, vals, vecs) < DENSE_EVD_QUALITY_THRESHOLD:
                return (vals, vecs), 0
        except SpectralError:
            pass
    if 1 not in skip_levels:
        r = lobpcg_solve(op, n_components, seed, False, sqrt_deg, stats=stats)
        if r is not None:
            (vals, vecs), _ = r
            if max_eigenpair_residual(lap, vals, vecs) < LOBPCG_QUALITY_THRESHOLD:
                return (vals, vecs), 1
    if 2 not in skip_levels:
        r = lobpcg_sinv_solve(lap, n_components, seed, sqrt_deg)
        if r is not None and max_eigenpair_residual(lap, *r) < SINV_LOBPCG_QUALITY_THRESHOLD:
            return r, 2
    if 3 not in skip_levels:
        r = lobpcg_solve(op, n_components, seed, True, sqrt_deg)
        if r is not None:
            (vals, vecs), _ = r
            if max_eigenpair_residual(lap, vals, vecs) < LOBPCG_QUALITY_THRESHOLD:
                return (vals, vecs), 3
    if 4 not in skip_levels:
        vals, vecs = rsvd_solve(lap, n_components, seed)
        if max_eigenpair_residual(lap, vals, vecs) < RSVD_QUALITY_THRESHOLD:
            return (vals, vecs), 4
    return dense_evd(lap, n_components + 1), 5


# --------------------------------------------------------------------------
# Selection, signs, scaling (src/selection.rs:11-29, src/scaling.rs:9-89)
# --------------------------------------------------------------------------
def select_eigenvectors(vals: np.ndarray, vecs: np.ndarray, n_components: int) -> np.ndarray:
    assert len(vals) > n_components, f"need at least n_components+1 eigenvalues, got {len(vals)}"
    order = sorted(range(len(vals)), key=lambda i: vals[i])  # stable, like sort_by
    return vecs[:, order[1:1 + n_components]].copy()


def normalize_signs(coords: np.ndarray) -> None:
    """Flip each column so its first largest-|.| element is positive
    (src/scaling.rs:62-74).

    The crate reduces with ``b.abs().total_cmp(&a.abs()).is_gt()``: on the
    non-negative |x| (sign bit clear) total_cmp is the order of the bit
    patterns as unsigned integers, so a NaN ranks above +inf (NaNs by payload)
    and ties keep the earlier row.  ``signum`` is -1 for negatives and -0.0
    and NaN for NaN, and only ``sign < 0`` flips, so a NaN maximum never flips.
    """
    for c in range(coords.shape[1]):
        col = np.ascontiguousarray(coords[:, c], dtype=np.float64)
        if col.size == 0:
            continue
        keys = col.view(np.uint64) & np.uint64(0x7FFFFFFFFFFFFFFF)
        i = int(np.argmax(keys))  # first maximum, like the strict-> reduce
        v = float(col[i])
        if not math.isnan(v) and math.copysign(1.0, v) < 0:
            coords[:, c] = -coords[:, c]


def scale_coords(coords: np.ndarray, max_coord: float) -> np.ndarray:
    max_abs = float(np.max(np.abs(coords))) if coords.size else 0.0
    if not max_abs > 0.0:
        raise InvalidGraph(f"scale_coords: embedding is all-zero; cannot scale to max={max_coord}")
    expansion = max_coord / max_abs
    return (coords * expansion).astype(np.float32)


def scale_and_add_noise(coords: np.ndarray, seed: int) -> np.ndarray:
    if coords.size == 0:
        raise InvalidGraph("scale_and_add_noise: input embedding is empty")
    scaled = scale_coords(coords, 10.0)
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(scaled.shape).astype(np.float32) * np.float32(1e-4)
    return scaled + noise


# --------------------------------------------------------------------------
# Multi-component layout (src/multi_component.rs:16-312)
# --------------------------------------------------------------------------
def collect_component_members(labels: np.ndarray, nc: int):
    members = [[] for _ in range(nc)]
    for node, lab in enumerate(labels):
        members[int(lab)].append(node)
    return [np.array(m, dtype=np.int64) for m in members]


def extract_subgraph(graph: sp.csr_matrix, nodes: np.ndarray) -> sp.csr_matrix:
    sub = graph[nodes][:, nodes]
    sub = sp.csr_matrix(sub, dtype=np.float32)
    sub.sort_indices()
    return sub


def orthogonal_meta_embedding(nc: int, dims: int) -> np.ndarray:
    m = np.zeros((nc, dims))
    for row in range(nc):
        m[row, row % dims] = 1.0 if row < dims else -1.0
    return m


def spectral_meta_embedding(data: np.ndarray, members, nc: int, dims: int, seed: int) -> np.ndarray:
    nf = data.shape[1]
    cent = np.zeros((nc, nf))
    for c, mem in enumerate(members):
        if len(mem) == 0:
            continue
        cent[c] = data[mem].astype(np.float64).sum(axis=0) * (1.0 / len(mem))
    d2 = ((cent[:, None, :] - cent[None, :, :]) ** 2).sum(axis=2)
    aff = np.exp(-d2)
    deg = np.array([sum(aff[i, j] for j in range(nc) if j != i) for i in range(nc)])
    inv = np.where(deg > 0, 1.0 / np.sqrt(np.where(deg > 0, deg, 1.0)), 0.0)
    lapd = np.eye(nc)
    for i in range(nc):
        for j in range(nc):
            if i != j:
                lapd[i, j] = -inv[i] * aff[i, j] * inv[j]
    lap = sp.csr_matrix(lapd)
    (vals, vecs), _ = solve_eigenproblem(lap, dims, seed, np.sqrt(deg))
    sel = select_eigenvectors(vals, vecs, dims)
    mx = float(np.max(np.abs(sel)))
    if mx == 0.0:
        raise InvalidGraph("spectral meta-embedding produced all-zero result")
    return sel / mx


def compute_data_range(meta: np.ndarray):
    nc = meta.shape[0]
    if nc == 1:
        return [1.0]
    out = []
    for c in range(nc):
        md = math.inf
        for i in range(nc):
            if i == c:
                continue
            dist = math.sqrt(float(((meta[c] - meta[i]) ** 2).sum()))
            if 0.0 < dist < md:
                md = dist
        out.append(md / 2.0 if math.isfinite(md) else 1.0)
    return out


def embed_single_component(graph, members, dims, data_range, meta_pos, seed, mode):
    size = len(members)
    if size < 2 * dims:
        return np.tile(meta_pos, (size, 1)).astype(np.float64)
    sub = extract_subgraph(graph, members)
    _, sqrt_deg = compute_degrees(sub, mode) if mode == PYTHON_COMPAT else compute_degrees_rust_native_fast(sub)
    lap = build_normalized_laplacian(sub, inv_sqrt(sqrt_deg))
    (vals, vecs), _ = solve_eigenproblem(lap, dims, seed, sqrt_deg)
    coords = select_eigenvectors(vals, vecs, dims)
    normalize_signs(coords)
    mx = float(np.max(np.abs(coords)))
    if mx > 0.0:
        coords *= data_range / mx
    return coords + meta_pos[None, :]


def embed_disconnected(graph, labels, nc, dims, seed, data=None, mode=PYTHON_COMPAT):
    n = graph.shape[0]
    members = collect_component_members(labels, nc)
    if nc > 2 * dims:
        if data is None:
            raise InvalidGraph("data is required for spectral meta-embedding when "
                               "n_conn_components > 2 * n_embedding_dims")
        meta = spectral_meta_embedding(np.asarray(data), members, nc, dims, seed)
    else:
        meta = orthogonal_meta_embedding(nc, dims)
    ranges = compute_data_range(meta)
    out = np.zeros((n, dims))
    for c, mem in enumerate(members):
        out[mem] = embed_single_component(graph, mem, dims, ranges[c], meta[c], seed, mode)
    return out


# --------------------------------------------------------------------------
# Pipeline (src/lib.rs:198-258)
# --------------------------------------------------------------------------
def spectral_init_prenoise(graph: sp.csr_matrix, n_components: int, seed: int, data=None,
                           mode: int = PYTHON_COMPAT):
    """Everything up to (not including) ``scale_and_add_noise``: returns the
    f64 coordinates that the crate hands to its final scaling step."""
    n = graph.shape[0]
    if n == 0 or n_components == 0:
        raise InvalidGraph(f"spectral_init requires n > 0 and n_components > 0; got n={n}, "
                           f"n_components={n_components}")
    if n <= n_components:
        raise TooFewNodes(n, n_components)
    labels, nc = find_components(graph) if n <= 20000 else find_components_fast(graph)
    if nc > 1:
        return embed_disconnected(graph, labels, nc, n_components, seed, data, mode)
    _, sqrt_deg = compute_degrees(graph, mode) if mode == PYTHON_COMPAT else compute_degrees_rust_native_fast(graph)
    lap = build_normalized_laplacian(graph, inv_sqrt(sqrt_deg))
    (vals, vecs), _ = solve_eigenproblem(lap, n_components, seed, sqrt_deg)
    sel = select_eigenvectors(vals, vecs, n_components)
    normalize_signs(sel)
    return sel


def spectral_init(graph: sp.csr_matrix, n_components: int, seed: int, data=None, mode: int = PYTHON_COMPAT):
    return scale_and_add_noise(spectral_init_prenoise(graph, n_components, seed, data, mode), seed)
