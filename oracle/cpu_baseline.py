"""Timed CPU restatement of the reference's eigensolve path (the CPU baseline).

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  The reference crate
is Rust and cannot be built here (no cargo/rustc, no vendored crates), so the
baseline is this port: the crate's LOBPCG wrapper (src/solvers/lobpcg.rs:
227-465, restated in ``spectral_oracle``) with the operator applied by the C
kernel ``csr_cpu.c`` (OpenMP over rows; AVX2 gather for single vectors, as in
src/operator.rs:96-145) and the dense block algebra in numpy/BLAS.

Recipe: ``build()`` compiles ``csr_cpu.c`` with ``gcc -O3 -mavx2 -mfma
-fopenmp`` into ``oracle/libcsr_cpu.so``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import time
from pathlib import Path

import numpy as np

from . import spectral_oracle as O

HERE = Path(__file__).resolve().parent
SRC = HERE / "csr_cpu.c"
LIB = HERE / "libcsr_cpu.so"
_lib = None


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    # AVX2 + FMA (the ISA of the crate's SIMD operator) rather than -march=native:
    # the library is built once and runs on other hosts' cores too
    cmd = ["gcc", "-O3", "-mavx2", "-mfma", "-fopenmp", "-shared", "-fPIC", str(SRC), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building csr_cpu.c failed:\n" + r.stderr)
    os.replace(tmp, LIB)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        lib.csr_spmm_f64.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_int]
        lib.csr_spmm_f64.restype = None
        lib.csr_threads.restype = C.c_int
        lib.csr_set_threads.argtypes = [C.c_int]
        lib.column_sum_f32.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def threads() -> int:
    return int(load().csr_threads())


class CpuOperator:
    """y = diag * x + V x with the C kernel (f64)."""

    def __init__(self, indptr, indices, data, n, diag=0.0):
        self.indptr = np.ascontiguousarray(indptr, dtype=np.uint64)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(data, dtype=np.float64)
        self.n = int(n)
        self.diag = float(diag)
        self.lib = load()
        self.applies = 0

    @staticmethod
    def from_csr(mat, diag=0.0):
        m = mat.tocsr()
        return CpuOperator(m.indptr, m.indices, m.data, m.shape[0], diag)

    def size(self):
        return self.n

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        k = 1 if x.ndim == 1 else x.shape[1]
        y = np.empty_like(x)
        self.lib.csr_spmm_f64(self.n, self.indptr.ctypes.data, self.indices.ctypes.data, self.data.ctypes.data,
                              self.diag, x.ctypes.data, y.ctypes.data, k)
        self.applies += 1
        return y


def time_spmm(op: CpuOperator, k: int, reps: int = 5) -> float:
    x = np.random.default_rng(0).standard_normal((op.n, k))
    op.apply(x)
    t = time.perf_counter()
    for _ in range(reps):
        op.apply(x)
    return (time.perf_counter() - t) / reps


def solve_timed(op: CpuOperator, n_components: int, seed: int, sqrt_deg, budget_s: float = 20.0,
                tol: float = O.LOBPCG_ACCEPT_TOL):
    """The crate's Level-1 solve (random start, Chebyshev filter, LOBPCG) on
    the CPU, stopped after ``budget_s`` seconds.  When it stops early the time
    to reach ``tol`` is projected from the log-linear decay of the largest
    wanted residual over the second half of the run."""
    n = op.size()
    k = n_components + 1
    t0 = time.perf_counter()
    x0 = O.initial_block(n, k, seed, np.asarray(sqrt_deg, dtype=np.float64))
    x0 = O.chebyshev_filter_start(op.apply, x0)
    t_filter = time.perf_counter() - t0
    hist = []
    t_start = time.perf_counter()

    def cb(it, rn):
        hist.append((time.perf_counter() - t_start, it, float(np.max(rn[:k]))))
        return (time.perf_counter() - t_start) > budget_s

    res = O.lobpcg_core(op.apply, x0, O.f32_tol(tol), min(5 * n, O.LOBPCG_INITIAL_MAXITER_CAP), callback=cb)
    t_iter_total = time.perf_counter() - t_start
    iters = max(res.iterations, 1)
    per_iter = t_iter_total / iters
    out = {"filter_s": t_filter, "iterations": res.iterations, "per_iteration_s": per_iter,
           "converged": bool(res.converged), "projected": False}
    if res.converged:
        out["seconds"] = t_filter + t_iter_total + 2 * time_spmm(op, k, 1)
        out["iterations_total"] = res.iterations
        return out
    tail = hist[len(hist) // 2:]
    if len(tail) >= 3:
        its = np.array([h[1] for h in tail], dtype=float)
        lr = np.log10(np.maximum([h[2] for h in tail], 1e-300))
        slope = np.polyfit(its, lr, 1)[0]
    else:
        slope = 0.0
    if slope < 0:
        need = its[-1] + (math.log10(tol) - lr[-1]) / slope
        out["iterations_total"] = float(need)
        out["seconds"] = t_filter + per_iter * need
        out["projected"] = True
    else:
        out["iterations_total"] = None
        out["seconds"] = t_filter + t_iter_total
        out["projected"] = "lower-bound"
    return out


def laplacian_operator(indptr, indices, weights, n: int):
    """The crate's Laplacian on the CPU (src/laplacian.rs:8-88): PythonCompat
    degrees by the f32 column scatter in CSR order, ``inv = 1/sqrt(d)`` (0 for
    isolated nodes), off-diagonal values ``-inv_i * w_ij * inv_j`` evaluated
    left to right in f64 on the graph's own pattern (self loops 0), unit
    diagonal applied implicitly.  Returns ``(CpuOperator, sqrt_deg)``."""
    ip = np.ascontiguousarray(indptr, dtype=np.uint64)
    ix = np.ascontiguousarray(indices, dtype=np.uint32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    deg = np.zeros(n, dtype=np.float32)
    load().column_sum_f32(len(ix), ix.ctypes.data, w.ctypes.data, deg.ctypes.data)
    sq = np.sqrt(deg.astype(np.float64))
    inv = O.inv_sqrt(sq)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ip.astype(np.int64)))
    cols = ix.astype(np.int64)
    vals = np.where(rows == cols, 0.0, (-inv[rows]) * w.astype(np.float64) * inv[cols])
    return CpuOperator(ip, ix, vals, n, diag=1.0), sq


def solve_measured(op: CpuOperator, n_components: int, seed: int, sqrt_deg):
    """The crate's Level-1 solve run to completion on the CPU and timed:
    seeded random start with the trivial-vector hint, Chebyshev filter,
    LOBPCG with warm restarts, Rayleigh-Ritz refinement and the per-vector
    residual check (src/solvers/lobpcg.rs:227-465), then the level gate
    (src/metrics.rs:73-92).  Nothing is projected."""
    stats = {}
    t0 = time.perf_counter()
    r = O.lobpcg_solve(op, n_components, seed, False, np.asarray(sqrt_deg, dtype=np.float64), stats=stats)
    gate = float("nan")
    if r is not None:
        (vals, vecs), _ = r
        lv = op.apply(vecs)
        d = lv - vecs * np.asarray(vals)[None, :]
        gate = float(np.max(np.linalg.norm(d, axis=0) / np.maximum(np.linalg.norm(vecs, axis=0), 1e-300)))
    secs = time.perf_counter() - t0
    return {"seconds": secs, "converged": r is not None and gate < O.LOBPCG_QUALITY_THRESHOLD,
            "iterations": stats.get("iterations"), "restarts": stats.get("restarts"), "max_residual": gate,
            "eigenvalues": None if r is None else [float(v) for v in r[0][0]]}


def set_threads(t: int) -> None:
    """Threads of the C kernels (OpenMP) and of numpy's BLAS."""
    load().csr_set_threads(int(t))
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(int(t))
    except Exception:
        pass
