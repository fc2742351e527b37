"""Certified FP64 eigenpairs of a normalised Laplacian: the accuracy oracle.

TEST INFRASTRUCTURE ONLY (the checker of ``tests/`` and of ``bench.py``'s
accuracy report; never the product path).

The reference crate (spectral-init) accepts an eigensolve when every residual
``||L v - lam v|| / ||v||`` is below its gate (src/metrics.rs:20-52, 57-92);
its own tests compare eigenvalues against ARPACK / dense ``eigh`` fixtures
(tests/generate_fixtures.py:256-326) and subspaces by the cross-Gram
determinant with degenerate pairs (gap < DEGENERATE_GAP_THRESHOLD = 1e-6,
src/metrics.rs:49) compared as subspaces (src/metrics.rs:212-288).  This
module supplies the exact side of such comparisons at any size:

* n <= ``DENSE_MAX``: dense LAPACK ``eigh`` of the matrix (exact to rounding);
* larger n: ARPACK (``scipy.sparse.linalg.eigsh``, implicitly restarted
  Lanczos) for the largest eigenvalues of ``2 I - L`` -- the smallest of L --
  run to machine precision, with ``k + extra`` pairs so that the gap to the
  first unwanted eigenvalue is known.

Every result carries its certificate: the FP64 residual of each pair,
recomputed here with an independent sparse product, and the Davis-Kahan bound
``sin(theta) <= residual / gap`` on the angle between each computed
eigenvector group and the exact eigenspace.  The bound assumes ARPACK found
the smallest eigenvalues (no eigenvalue below the returned ones is missed);
the returned set is the ``k + extra`` smallest with a margin of ``extra``
pairs, and a solver under test that found a smaller eigenvalue would show up
as a failed comparison, not a pass.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

DENSE_MAX = 6000
DEGENERATE_GAP_THRESHOLD = 1e-6  # src/metrics.rs:49


@dataclass
class Reference:
    vals: np.ndarray          # ascending, k + extra (or all, dense)
    vecs: np.ndarray          # [n, len(vals)], orthonormal columns
    residuals: np.ndarray     # FP64 residual per pair
    method: str
    extra: int = 0
    notes: dict = field(default_factory=dict)


def laplacian_from_operator(indptr, indices, values, n: int, diag: float = 1.0) -> sp.csr_matrix:
    """Explicit f64 CSR ``diag * I + V`` of an implicit-diagonal operator
    (stored entries ``values`` on the pattern ``indptr``/``indices``)."""
    v = sp.csr_matrix((np.asarray(values, np.float64), np.asarray(indices, np.int64),
                       np.asarray(indptr, np.int64)), shape=(n, n))
    return (v + diag * sp.identity(n, format="csr", dtype=np.float64)).tocsr()


def residuals(lap: sp.csr_matrix, vals: np.ndarray, vecs: np.ndarray) -> np.ndarray:
    """``||L v_i - lam_i v_i|| / ||v_i||`` in FP64 (src/metrics.rs:57-72)."""
    lv = lap @ vecs
    d = lv - vecs * np.asarray(vals)[None, :]
    return np.linalg.norm(d, axis=0) / np.maximum(np.linalg.norm(vecs, axis=0), 1e-300)


def reference_eigenpairs(lap: sp.csr_matrix, k: int, extra: int = 6, dense_max: int = DENSE_MAX) -> Reference:
    """The ``k + extra`` smallest eigenpairs of the symmetric ``lap`` in FP64."""
    n = lap.shape[0]
    m = min(n, k + extra)
    if n <= dense_max:
        w, v = np.linalg.eigh(lap.toarray())
        vals, vecs, method = w[:m].copy(), v[:, :m].copy(), "dense LAPACK eigh (numpy)"
    else:
        shifted = (2.0 * sp.identity(n, format="csr", dtype=np.float64) - lap).tocsr()
        ncv = min(n - 1, max(2 * m + 1, 48))
        w, v = sla.eigsh(shifted, k=m, which="LA", tol=0.0, ncv=ncv, maxiter=max(1000, 20 * n // ncv))
        order = np.argsort(-w, kind="stable")
        vals = 2.0 - w[order]
        vecs = v[:, order]
        method = f"ARPACK eigsh on 2I-L (k={m}, ncv={ncv}, tol=machine precision)"
    res = residuals(lap, vals, vecs)
    return Reference(vals=vals, vecs=vecs, residuals=res, method=method, extra=m - k)


def reference_eigenpairs_operator(apply_l, n: int, k: int, extra: int = 6) -> Reference:
    """As ``reference_eigenpairs`` for an operator given only by its product
    ``apply_l(x) = L x`` (1-D or row-major 2-D ``x``; e.g. the multi-threaded
    C CSR kernel of ``cpu_baseline``): ARPACK on ``2 I - L``."""
    m = min(n - 1, k + extra)
    shifted = sla.LinearOperator((n, n), matvec=lambda v: 2.0 * v - apply_l(np.ascontiguousarray(v).ravel()),
                                 dtype=np.float64)
    ncv = min(n - 1, max(2 * m + 1, 48))
    w, v = sla.eigsh(shifted, k=m, which="LA", tol=0.0, ncv=ncv, maxiter=max(1000, 20 * n // ncv))
    order = np.argsort(-w, kind="stable")
    vals = 2.0 - w[order]
    vecs = np.ascontiguousarray(v[:, order])
    lv = apply_l(vecs)
    d = lv - vecs * vals[None, :]
    res = np.linalg.norm(d, axis=0) / np.maximum(np.linalg.norm(vecs, axis=0), 1e-300)
    return Reference(vals=vals, vecs=vecs, residuals=res, extra=m - k,
                     method=f"ARPACK eigsh on 2I-L (k={m}, ncv={ncv}, tol=machine precision)")


def degenerate_groups(vals: np.ndarray, thr: float = DEGENERATE_GAP_THRESHOLD):
    """Maximal runs of consecutive eigenvalues whose neighbours are closer than ``thr``."""
    groups, cur = [], [0]
    for i in range(1, len(vals)):
        if vals[i] - vals[i - 1] < thr:
            cur.append(i)
        else:
            groups.append(cur)
            cur = [i]
    groups.append(cur)
    return groups


def _orth(a: np.ndarray) -> np.ndarray:
    return np.linalg.qr(a)[0]


def sin_theta_into(a: np.ndarray, b: np.ndarray) -> float:
    """Largest principal-angle sine of span(a) against span(b) (dim a <= dim b):
    ``||(I - Qb Qb^T) Qa||_2``, accurate for tiny angles."""
    qa = _orth(a)
    qb = _orth(b)
    return float(np.linalg.norm(qa - qb @ (qb.T @ qa), 2))


def compare(vals: np.ndarray, vecs: np.ndarray, ref: Reference, wanted=None, thr: float = DEGENERATE_GAP_THRESHOLD):
    """Errors of computed eigenpairs (``vals`` ascending, ``vecs`` [n, k])
    against the reference, per result:

    * ``eig_rel``: |lam_i - lam_i^ref| / |lam_i^ref| for the wanted indices
      (``wanted`` defaults to 1..k-1, the nontrivial pairs; index 0 is the
      trivial eigenvalue, compared absolutely in ``eig_abs0``);
    * ``sin_theta``: per degenerate group of the reference (gap < ``thr``),
      the largest principal-angle sine of the computed vectors of the group
      against the reference eigenspace of the whole group (rotation- and
      sign-invariant), and ``sin_theta_max`` over groups;
    * ``sin_theta_subspace``: the same for all wanted vectors at once against
      the reference span of every group they touch;
    * ``oracle_sin_theta_bound``: the Davis-Kahan bound residual / gap of the
      reference itself (how exact the oracle is).
    """
    vals = np.asarray(vals, np.float64)
    k = len(vals)
    if wanted is None:
        wanted = list(range(1, k))
    rv = ref.vals
    if len(rv) < k:
        raise ValueError("reference has fewer pairs than the result")
    groups = degenerate_groups(rv, thr)
    gid = {i: gi for gi, g in enumerate(groups) for i in g}
    out = {"method": ref.method}
    out["eig_rel"] = [float(abs(vals[i] - rv[i]) / max(abs(rv[i]), 1e-300)) for i in wanted]
    out["eig_rel_max"] = max(out["eig_rel"]) if wanted else 0.0
    out["eig_abs0"] = float(abs(vals[0] - rv[0]))
    per_group = []
    touched = sorted({gid[i] for i in wanted})
    for gi in touched:
        idx = [i for i in wanted if gid[i] == gi]
        g = groups[gi]
        if g[-1] == len(rv) - 1 and len(rv) < ref.vecs.shape[0]:
            raise ValueError("a wanted degenerate group reaches the end of the reference set; "
                             "ask the oracle for more pairs (extra)")
        per_group.append({"indices": idx, "group": [int(g[0]), int(g[-1])],
                          "sin_theta": sin_theta_into(vecs[:, idx], ref.vecs[:, g])})
    out["groups"] = per_group
    out["sin_theta_max"] = max(p["sin_theta"] for p in per_group) if per_group else 0.0
    span = sorted({j for gi in touched for j in groups[gi]})
    out["sin_theta_subspace"] = sin_theta_into(vecs[:, wanted], ref.vecs[:, span]) if wanted else 0.0
    bounds = []
    for gi in touched:
        g = groups[gi]
        lo = rv[g[0] - 1] if g[0] > 0 else -math.inf
        hi = rv[g[-1] + 1] if g[-1] + 1 < len(rv) else math.inf
        gap = min(rv[g[0]] - lo, hi - rv[g[-1]])
        bounds.append(float(np.max(ref.residuals[g]) / gap) if gap > 0 else math.inf)
    out["oracle_sin_theta_bound"] = max(bounds) if bounds else 0.0
    out["oracle_max_residual"] = float(np.max(ref.residuals[: max(k, 1)]))
    return out


def gap_after(ref: Reference, k: int) -> float:
    """lam_k - lam_{k-1} of the reference: the gap that bounds the angle of the
    first k eigenvectors (residual / gap)."""
    return float(ref.vals[k] - ref.vals[k - 1])
