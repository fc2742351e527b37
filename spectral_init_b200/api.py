"""Python mirror of the spectral-init crate's API over the sm_100a C ABI.

Names, argument meaning and error behaviour follow the crate:
``spectral_init`` (src/lib.rs:198-258), ``SpectralInitConfig`` / ``ComputeMode``
(src/config.rs:5-25), ``SpectralError`` (src/lib.rs:167-182) and the
component-level seams re-exported by src/lib.rs:20-162
(``compute_degrees``, ``build_normalized_laplacian``, ``find_components``,
``solve_eigenproblem_pub``, ``lobpcg_solve``, ``rsvd_solve``, ``dense_evd``,
``select_eigenvectors``, ``normalize_signs_pub``, ``scale_and_add_noise_pub``).

All numerical work runs in ``libspectral_init_b200.so``; host arrays are staged
to the device by the library itself (``spectral_init`` and the ``*_host``
entry points) or through torch CUDA tensors for the device-pointer entry
points.  There is no CPU fallback: without the library every call raises.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import SiConfig, SiCsrF32, SiCsrF64, SiOperator, SiReport


class ComputeMode(IntEnum):
    """src/config.rs:5-14."""
    PythonCompat = 0
    RustNative = 1


class Precision(IntEnum):
    FP64 = 0
    MIXED = 1


class WarmStart(IntEnum):
    RANDOM = 0
    LEARNED = 1


@dataclass
class SpectralInitConfig:
    """``SpectralInitConfig`` (src/config.rs:21-25) plus the device solver policy."""
    compute_mode: ComputeMode = ComputeMode.PythonCompat
    precision: Precision = Precision.FP64
    warm_start: WarmStart = WarmStart.RANDOM
    block_size: int = 0
    dense_threshold: int = 0
    force_level: int = -1
    rsvd_oversampling: int = -1
    rsvd_nbiter: int = 0
    max_iterations: int = 0
    learned_filter: int = 0
    tol: float = 0.0
    mixed_switch_tol: float = 0.0

    def to_c(self) -> SiConfig:
        c = SiConfig()
        _lib.load().si_config_default(C.byref(c))
        for f in ("compute_mode", "precision", "warm_start", "block_size", "dense_threshold", "force_level",
                  "rsvd_oversampling", "rsvd_nbiter", "max_iterations", "learned_filter"):
            setattr(c, f, int(getattr(self, f)))
        c.tol = float(self.tol)
        c.mixed_switch_tol = float(self.mixed_switch_tol)
        return c


# ---- errors (src/lib.rs:167-182) ---------------------------------------------------
class SpectralError(Exception):
    code = -1


class ConvergenceFailure(SpectralError):
    code = _lib.SI_CONVERGENCE_FAILURE


class InvalidGraph(SpectralError):
    code = _lib.SI_INVALID_GRAPH


class TooFewNodes(SpectralError):
    code = _lib.SI_TOO_FEW_NODES

    def __init__(self, msg, n=None, dims=None):
        super().__init__(msg)
        self.n = n
        self.dims = dims


class CudaError(SpectralError):
    code = _lib.SI_CUDA_ERROR


class IterationCap(SpectralError):
    code = _lib.SI_ITERATION_CAP


class InvalidArgument(SpectralError, ValueError):
    code = _lib.SI_INVALID_ARGUMENT


class OutOfMemory(SpectralError, MemoryError):
    code = _lib.SI_OUT_OF_MEMORY


_ERRORS = {c.code: c for c in (ConvergenceFailure, InvalidGraph, TooFewNodes, CudaError, IterationCap,
                               InvalidArgument, OutOfMemory)}


@dataclass
class Report:
    level: int = -1
    iterations: int = 0
    restarts: int = 0
    n_components_graph: int = 0
    fp32_iterations: int = 0
    spmm_calls: int = 0
    max_residual: float = 0.0
    solve_ms: float = 0.0
    eigenvalues: list = field(default_factory=list)
    learned_start: int = 0

    @staticmethod
    def from_c(r: SiReport, k: int) -> "Report":
        return Report(r.level, r.iterations, r.restarts, r.n_components_graph, r.fp32_iterations, r.spmm_calls,
                      r.max_residual, r.solve_ms, [r.eigenvalues[i] for i in range(min(k, 16))],
                      r.learned_start)


# ---- context -------------------------------------------------------------------------
class Context:
    """One CUDA stream + workspace on one device (``si_ctx``)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        self.ptr = C.c_void_p()
        st = self.lib.si_ctx_create(int(device), C.byref(self.ptr))
        if st != _lib.SI_OK:
            raise CudaError(f"si_ctx_create(device={device}) failed with status {st}")
        self.device = device

    def check(self, status: int, n=None, dims=None):
        if status == _lib.SI_OK:
            return
        msg = (self.lib.si_last_error(self.ptr) or b"").decode(errors="replace")
        cls = _ERRORS.get(status, SpectralError)
        if cls is TooFewNodes:
            raise TooFewNodes(msg, n, dims)
        raise cls(msg)

    def synchronize(self):
        self.check(self.lib.si_ctx_synchronize(self.ptr))

    def close(self):
        if self.ptr:
            self.lib.si_ctx_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


def get_context(device: int = 0) -> Context:
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


# ---- host array helpers ------------------------------------------------------------------
def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


def as_csr_f32(graph):
    """(n, indptr u64, indices u32, data f32) from a scipy sparse matrix or a
    (indptr, indices, data, n) tuple -- the crate's CsMatI<f32, u32, usize>."""
    if isinstance(graph, tuple):
        indptr, indices, data, n = graph
    else:
        g = graph.tocsr()
        indptr, indices, data, n = g.indptr, g.indices, g.data, g.shape[0]
        if g.shape[0] != g.shape[1]:
            raise InvalidGraph(f"invalid graph: adjacency matrix must be square, got {g.shape}")
    indptr = np.ascontiguousarray(indptr, dtype=np.uint64)
    indices = np.ascontiguousarray(indices, dtype=np.uint32)
    data = np.ascontiguousarray(data, dtype=np.float32)
    return int(n), indptr, indices, data


def as_csr_f64(mat):
    if isinstance(mat, tuple):
        indptr, indices, data, n = mat
    else:
        m = mat.tocsr()
        m.sort_indices()
        indptr, indices, data, n = m.indptr, m.indices, m.data, m.shape[0]
    return (int(n), np.ascontiguousarray(indptr, dtype=np.uint64), np.ascontiguousarray(indices, dtype=np.uint32),
            np.ascontiguousarray(data, dtype=np.float64))


def _c_csr32(n, indptr, indices, data) -> SiCsrF32:
    return SiCsrF32(n, int(indices.size), _ptr(indptr).value, _ptr(indices).value, _ptr(data).value)


def _c_csr64(n, indptr, indices, data) -> SiCsrF64:
    return SiCsrF64(n, int(indices.size), _ptr(indptr).value, _ptr(indices).value, _ptr(data).value)


# ---- pipeline ---------------------------------------------------------------------------------
def spectral_init(graph, n_components: int, seed: int, data=None, config: SpectralInitConfig | None = None, *,
                  ctx: Context | None = None, return_report: bool = False):
    """spectral_init (src/lib.rs:198-258) on the GPU.  Returns f32 [n, n_components]."""
    ctx = ctx or get_context()
    cfg = (config or SpectralInitConfig()).to_c()
    n, indptr, indices, vals = as_csr_f32(graph)
    out = np.zeros((n, max(int(n_components), 0)), dtype=np.float32)
    dptr, nf = C.c_void_p(0), 0
    if data is not None:
        d = np.ascontiguousarray(data, dtype=np.float32)
        dptr, nf = _ptr(d), d.shape[1]
    rep = SiReport()
    st = ctx.lib.si_spectral_init(ctx.ptr, C.byref(_c_csr32(n, indptr, indices, vals)), int(n_components),
                                  int(seed) & 0xFFFFFFFFFFFFFFFF, dptr, nf, C.byref(cfg), _ptr(out), C.byref(rep))
    ctx.check(st, n, n_components)
    if return_report:
        return out, Report.from_c(rep, n_components + 1)
    return out


# ---- component seams (host in / host out) ------------------------------------------------------
def _torch():
    import torch  # noqa: WPS433 -- device staging only
    if not torch.cuda.is_available():
        raise CudaError("no CUDA device available")
    return torch


class _DevGraph:
    """Graph staged in device memory via torch (plumbing for the device-pointer entry points)."""

    def __init__(self, graph, device=0):
        torch = _torch()
        self.n, indptr, indices, data = as_csr_f32(graph)
        dev = torch.device("cuda", device)
        self.indptr = torch.from_numpy(indptr.view(np.int64)).to(dev)
        self.indices = torch.from_numpy(indices.view(np.int32)).to(dev)
        self.data = torch.from_numpy(data).to(dev)
        self.nnz = int(indices.size)
        torch.cuda.synchronize(dev)

    def c(self) -> SiCsrF32:
        return SiCsrF32(self.n, self.nnz, self.indptr.data_ptr(), self.indices.data_ptr() if self.nnz else 0,
                        self.data.data_ptr() if self.nnz else 0)


def compute_degrees(graph, mode: ComputeMode = ComputeMode.PythonCompat, *, ctx: Context | None = None):
    """compute_degrees (src/laplacian.rs:29-49) -> (degrees, sqrt_deg) f64."""
    ctx = ctx or get_context()
    torch = _torch()
    g = _DevGraph(graph, ctx.device)
    deg = torch.empty(max(g.n, 1), dtype=torch.float64, device=f"cuda:{ctx.device}")
    sq = torch.empty_like(deg)
    ctx.check(ctx.lib.si_compute_degrees(ctx.ptr, C.byref(g.c()), int(mode), deg.data_ptr(), sq.data_ptr()))
    return deg[:g.n].cpu().numpy(), sq[:g.n].cpu().numpy()


def build_laplacian_values(graph, inv_sqrt_deg, *, ctx: Context | None = None, with_f32: bool = False):
    """Implicit-diagonal Laplacian values (one per stored graph entry)."""
    ctx = ctx or get_context()
    torch = _torch()
    g = _DevGraph(graph, ctx.device)
    dev = f"cuda:{ctx.device}"
    inv = torch.from_numpy(np.ascontiguousarray(inv_sqrt_deg, dtype=np.float64)).to(dev)
    v64 = torch.empty(max(g.nnz, 1), dtype=torch.float64, device=dev)
    v32 = torch.empty(max(g.nnz, 1), dtype=torch.float32, device=dev) if with_f32 else None
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_build_laplacian(ctx.ptr, C.byref(g.c()), inv.data_ptr(), v64.data_ptr(),
                                         v32.data_ptr() if v32 is not None else None))
    out64 = v64[:g.nnz].cpu().numpy()
    return (out64, v32[:g.nnz].cpu().numpy()) if with_f32 else out64


def build_normalized_laplacian(graph, inv_sqrt_deg, *, ctx: Context | None = None):
    """build_normalized_laplacian (src/laplacian.rs:60-88) -> scipy CSR f64 with
    sorted columns and the unit diagonal, exactly as the crate returns it."""
    import scipy.sparse as sp
    ctx = ctx or get_context()
    torch = _torch()
    g = _DevGraph(graph, ctx.device)
    dev = f"cuda:{ctx.device}"
    inv = torch.from_numpy(np.ascontiguousarray(inv_sqrt_deg, dtype=np.float64)).to(dev)
    torch.cuda.synchronize()
    nnz = C.c_uint64(0)
    ctx.check(ctx.lib.si_build_laplacian_csr(ctx.ptr, C.byref(g.c()), inv.data_ptr(), None, None, None,
                                             C.byref(nnz)))
    ip = torch.empty(g.n + 1, dtype=torch.int64, device=dev)
    ix = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
    dv = torch.empty(max(nnz.value, 1), dtype=torch.float64, device=dev)
    ctx.check(ctx.lib.si_build_laplacian_csr(ctx.ptr, C.byref(g.c()), inv.data_ptr(), ip.data_ptr(),
                                             ix.data_ptr(), dv.data_ptr(), C.byref(nnz)))
    k = nnz.value
    return sp.csr_matrix((dv[:k].cpu().numpy(), ix[:k].cpu().numpy().view(np.uint32).astype(np.int64),
                          ip.cpu().numpy()), shape=(g.n, g.n))


def fuzzy_graph(points, k: int = 15, *, ctx: Context | None = None, return_stages: bool = False):
    """The fuzzy-kNN graph of ``points`` ([n, dims]) on the device, as the
    crate's fixture generator builds it (tests/generate_fixtures.py:70-182):
    exact kNN without the point itself, umap-learn's smooth-kNN, membership
    strengths, fuzzy union, pruning.  Returns the scipy CSR (f32), and with
    ``return_stages`` also (knn_indices, knn_dists, sigmas, rhos)."""
    import scipy.sparse as sp
    ctx = ctx or get_context()
    torch = _torch()
    dev = f"cuda:{ctx.device}"
    x = torch.as_tensor(np.ascontiguousarray(points, dtype=np.float64), device=dev)
    n, d = x.shape
    cap = 2 * n * k
    idx = torch.empty(n, k, dtype=torch.int32, device=dev)
    dist = torch.empty(n, k, dtype=torch.float32, device=dev)
    sig = torch.empty(n, dtype=torch.float32, device=dev)
    rho = torch.empty(n, dtype=torch.float32, device=dev)
    ip = torch.empty(n + 1, dtype=torch.int64, device=dev)
    ix = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
    dv = torch.empty(max(cap, 1), dtype=torch.float32, device=dev)
    nnz = C.c_uint64(0)
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_fuzzy_graph(ctx.ptr, x.data_ptr(), n, d, k, idx.data_ptr(), dist.data_ptr(), sig.data_ptr(),
                                     rho.data_ptr(), ip.data_ptr(), ix.data_ptr(), dv.data_ptr(), cap,
                                     C.byref(nnz)))
    m = int(nnz.value)
    g = sp.csr_matrix((dv[:m].cpu().numpy(), ix[:m].cpu().numpy(), ip.cpu().numpy()), shape=(n, n))
    if return_stages:
        return g, (idx.cpu().numpy(), dist.cpu().numpy(), sig.cpu().numpy(), rho.cpu().numpy())
    return g


def find_components(graph, *, ctx: Context | None = None):
    """find_components (src/components.rs:7-44) -> (labels, n_components)."""
    ctx = ctx or get_context()
    torch = _torch()
    g = _DevGraph(graph, ctx.device)
    labels = torch.empty(max(g.n, 1), dtype=torch.int32, device=f"cuda:{ctx.device}")
    nc = C.c_uint64(0)
    ctx.check(ctx.lib.si_find_components(ctx.ptr, C.byref(g.c()), labels.data_ptr(), C.byref(nc)))
    return labels[:g.n].cpu().numpy().astype(np.int64), int(nc.value)


def solve_eigenproblem_pub(laplacian, n_components: int, seed: int, config: SpectralInitConfig | None = None, *,
                           ctx: Context | None = None, return_report: bool = False):
    """solve_eigenproblem_pub (src/lib.rs:67-75) -> ((vals, vecs), level)."""
    ctx = ctx or get_context()
    n, ip, ix, dv = as_csr_f64(laplacian)
    k = n_components + 1
    vals = np.zeros(k)
    vecs = np.zeros((n, k))
    level = C.c_int32(-1)
    rep = SiReport()
    cfg = (config or SpectralInitConfig()).to_c()
    ctx.check(ctx.lib.si_solve_eigenproblem_host(ctx.ptr, C.byref(_c_csr64(n, ip, ix, dv)), int(n_components),
                                                 int(seed), C.byref(cfg), _ptr(vals), _ptr(vecs), C.byref(level),
                                                 C.byref(rep)), n, n_components)
    res = ((vals, vecs), int(level.value))
    return (res, Report.from_c(rep, k)) if return_report else res


def lobpcg_solve(laplacian, n_components: int, seed: int, regularize: bool, sqrt_deg,
                 config: SpectralInitConfig | None = None, *, ctx: Context | None = None,
                 return_report: bool = False):
    """lobpcg_solve (src/solvers/lobpcg.rs:227-465) -> ((vals, vecs), restarts) or None."""
    ctx = ctx or get_context()
    n, ip, ix, dv = as_csr_f64(laplacian)
    k = n_components + 1
    if n_components == 0 or k >= n or len(sqrt_deg) != n:
        return None
    sq = np.ascontiguousarray(sqrt_deg, dtype=np.float64)
    vals = np.zeros(k)
    vecs = np.zeros((n, k))
    restarts = C.c_int32(0)
    rep = SiReport()
    cfg = (config or SpectralInitConfig()).to_c()
    st = ctx.lib.si_lobpcg_solve_host(ctx.ptr, C.byref(_c_csr64(n, ip, ix, dv)), int(n_components), int(seed),
                                      int(bool(regularize)), _ptr(sq), C.byref(cfg), _ptr(vals), _ptr(vecs),
                                      C.byref(restarts), C.byref(rep))
    if st == _lib.SI_CONVERGENCE_FAILURE:
        return None
    ctx.check(st)
    res = ((vals, vecs), int(restarts.value))
    return (res, Report.from_c(rep, k)) if return_report else res


def rsvd_solve(laplacian, n_components: int, seed: int, oversampling: int | None = None,
               nbiter: int | None = None, *, ctx: Context | None = None):
    """rsvd_solve (src/solvers/rsvd.rs:135-213) -> (vals, vecs)."""
    ctx = ctx or get_context()
    n, ip, ix, dv = as_csr_f64(laplacian)
    k = n_components + 1
    vals = np.zeros(k)
    vecs = np.zeros((n, k))
    ctx.check(ctx.lib.si_rsvd_solve_host(ctx.ptr, C.byref(_c_csr64(n, ip, ix, dv)), int(n_components), int(seed),
                                         -1 if oversampling is None else int(oversampling),
                                         0 if nbiter is None else int(nbiter), _ptr(vals), _ptr(vecs)))
    return vals, vecs


def dense_evd(laplacian, k: int, *, ctx: Context | None = None):
    """dense_evd (src/solvers/dense.rs:9-46) -> (vals[k], vecs[n, k])."""
    ctx = ctx or get_context()
    n, ip, ix, dv = as_csr_f64(laplacian)
    vals = np.zeros(k)
    vecs = np.zeros((n, k))
    ctx.check(ctx.lib.si_dense_evd_host(ctx.ptr, C.byref(_c_csr64(n, ip, ix, dv)), int(k), _ptr(vals),
                                        _ptr(vecs)), n, k)
    return vals, vecs


def select_eigenvectors(eigenvalues, eigenvectors, n_components: int):
    """select_eigenvectors (src/selection.rs:11-29): argsort ascending, skip index 0."""
    ev = np.asarray(eigenvalues)
    if len(ev) <= n_components:
        raise AssertionError(f"need at least n_components+1 eigenvalues, got {len(ev)}")
    order = sorted(range(len(ev)), key=lambda i: ev[i])
    return np.asarray(eigenvectors)[:, order[1:1 + n_components]].copy()


def normalize_signs(coords, *, ctx: Context | None = None):
    """normalize_signs (src/scaling.rs:62-74) on the device; returns the flipped copy."""
    ctx = ctx or get_context()
    torch = _torch()
    x = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.float64)).to(f"cuda:{ctx.device}")
    torch.cuda.synchronize()
    n, k = x.shape
    ctx.check(ctx.lib.si_normalize_signs(ctx.ptr, x.data_ptr(), n, k))
    return x.cpu().numpy()


def scale_and_add_noise(coords, seed: int, *, ctx: Context | None = None):
    """scale_and_add_noise (src/scaling.rs:78-89) on the device -> f32."""
    ctx = ctx or get_context()
    torch = _torch()
    c = np.ascontiguousarray(coords, dtype=np.float64)
    if c.size == 0:
        raise InvalidGraph("scale_and_add_noise: input embedding is empty")
    x = torch.from_numpy(c).to(f"cuda:{ctx.device}")
    out = torch.empty(c.shape, dtype=torch.float32, device=f"cuda:{ctx.device}")
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_scale_and_add_noise(ctx.ptr, x.data_ptr(), c.shape[0], c.shape[1], int(seed),
                                             out.data_ptr()))
    return out.cpu().numpy()


class CsrOperator:
    """``LinearOperator`` (src/operator.rs:7-12) over a device CSR operator:
    ``apply(x)`` returns ``diag * x + V x`` for torch CUDA blocks [n, k]."""

    def __init__(self, laplacian, diag: float = 0.0, *, ctx: Context | None = None, with_f32: bool = False):
        self.ctx = ctx or get_context()
        torch = _torch()
        n, ip, ix, dv = as_csr_f64(laplacian)
        dev = f"cuda:{self.ctx.device}"
        self.n = n
        self.indptr = torch.from_numpy(ip.view(np.int64)).to(dev)
        self.indices = torch.from_numpy(ix.view(np.int32)).to(dev)
        self.values = torch.from_numpy(dv).to(dev)
        self.values32 = self.values.float() if with_f32 else None
        self.diag = float(diag)
        torch.cuda.synchronize()

    def c(self) -> SiOperator:
        return SiOperator(self.n, int(self.indices.numel()), self.indptr.data_ptr(), self.indices.data_ptr(),
                          self.values.data_ptr(),
                          self.values32.data_ptr() if self.values32 is not None else None, self.diag)

    def size(self) -> int:
        return self.n

    def apply(self, x):
        torch = _torch()
        x = x.contiguous()
        y = torch.empty_like(x)
        k = x.shape[1] if x.dim() == 2 else 1
        torch.cuda.synchronize()
        if x.dtype == torch.float64:
            self.ctx.check(self.ctx.lib.si_spmm(self.ctx.ptr, C.byref(self.c()), x.data_ptr(), y.data_ptr(), k))
        else:
            self.ctx.check(self.ctx.lib.si_spmm_f32(self.ctx.ptr, C.byref(self.c()), x.data_ptr(), y.data_ptr(), k))
        return y

    # ---- prepared operator (si_operator_plan): repeated products without per-call set-up ----
    def prepare(self) -> "CsrOperator":
        """Build the operator's plan once (row partitions, panel windows on
        first use of each width); ``apply_prepared`` then reuses it."""
        if getattr(self, "_plan", None) is None:
            h = C.c_void_p()
            self.ctx.check(self.ctx.lib.si_operator_plan_create(self.ctx.ptr, C.byref(self.c()), C.byref(h)))
            self._plan = h
        return self

    def apply_prepared(self, x, y=None):
        """``y = diag * x + V x`` through the prepared operator, queued on the
        library's stream without waiting (``ctx.synchronize()`` waits)."""
        torch = _torch()
        self.prepare()
        x = x.contiguous()
        if y is None:
            y = torch.empty_like(x)
        k = x.shape[1] if x.dim() == 2 else 1
        fn = self.ctx.lib.si_spmm_planned if x.dtype == torch.float64 else self.ctx.lib.si_spmm_planned_f32
        self.ctx.check(fn(self.ctx.ptr, self._plan, x.data_ptr(), y.data_ptr(), k))
        return y

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None:
            self.ctx.lib.si_operator_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
