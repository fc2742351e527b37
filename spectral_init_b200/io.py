"""CSR graph files and embedding output for end-to-end runs.

The crate's consumers hand ``spectral_init`` a ``CsMatI<f32, u32, usize>``
fuzzy-kNN graph; its tests read graphs and Laplacians from scipy's sparse
``.npz`` format (tests/common/mod.rs:30-80 of the reference: ``data`` as f64
or f32, ``indices`` / ``indptr`` as i32 or i64, ``shape``).  This module reads
and writes that format with the same tolerance for index and value types, and
runs the device pipeline from a file:

    python -m spectral_init_b200.io graph.npz embedding.npy [--n-components 2]
        [--seed 42] [--data points.npy] [--precision fp64|mixed]

Nothing here computes: the embedding comes from ``spectral_init`` (the CUDA
library).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

from .api import InvalidGraph


def _read(z, key):
    if key not in z.files:
        raise InvalidGraph(f"npz graph: missing array '{key}'")
    return z[key]


def load_csr_npz(path, value_dtype=np.float32) -> sp.csr_matrix:
    """A scipy-format CSR ``.npz`` as a sorted ``csr_matrix`` with
    ``value_dtype`` values (f32 for graphs, f64 for Laplacians) and int32/int64
    index arrays as stored.  Malformed files raise ``InvalidGraph``."""
    with np.load(path, allow_pickle=False) as z:
        fmt = z["format"].item() if "format" in z.files else b"csr"
        fmt = fmt.decode() if isinstance(fmt, bytes) else str(fmt)
        if fmt != "csr":
            raise InvalidGraph(f"npz graph: format '{fmt}', expected 'csr'")
        data = _read(z, "data")
        indices = _read(z, "indices")
        indptr = _read(z, "indptr")
        shape = tuple(int(v) for v in _read(z, "shape"))
    if len(shape) != 2 or shape[0] != shape[1]:
        raise InvalidGraph(f"npz graph: shape {shape} is not square")
    n = shape[0]
    if data.dtype not in (np.float32, np.float64):
        raise InvalidGraph(f"npz graph: data dtype {data.dtype}, expected f32 or f64")
    if indices.dtype not in (np.int32, np.int64, np.uint32, np.uint64) or indptr.dtype not in (np.int32, np.int64,
                                                                                               np.uint64):
        raise InvalidGraph("npz graph: indices / indptr must be 32- or 64-bit integers")
    if indptr.ndim != 1 or len(indptr) != n + 1 or int(indptr[0]) != 0 or int(indptr[-1]) != len(indices) \
            or len(indices) != len(data) or np.any(np.diff(indptr.astype(np.int64)) < 0):
        raise InvalidGraph(f"npz graph: inconsistent CSR arrays (n={n}, indptr {len(indptr)}, "
                           f"indices {len(indices)}, data {len(data)})")
    if len(indices) and (int(indices.min()) < 0 or int(indices.max()) >= n):
        raise InvalidGraph("npz graph: column index out of range")
    g = sp.csr_matrix((data.astype(value_dtype, copy=False), indices, indptr), shape=(n, n))
    if not g.has_sorted_indices:
        g = g.copy()
        g.sort_indices()
    return g


def save_csr_npz(path, graph) -> None:
    """Write ``graph`` (any scipy sparse matrix) in scipy's CSR ``.npz`` layout
    (the format ``scipy.sparse.save_npz`` writes and ``load_csr_npz`` reads)."""
    g = sp.csr_matrix(graph)
    g.sort_indices()
    idx_t = np.int32 if g.nnz < 2**31 and g.shape[0] < 2**31 else np.int64
    np.savez(path, data=g.data, indices=g.indices.astype(idx_t), indptr=g.indptr.astype(idx_t),
             format=np.array(b"csr"), shape=np.array(g.shape, dtype=np.int64))


def save_embedding(path, embedding) -> None:
    """The ``[n, n_components]`` f32 embedding as ``.npy``."""
    np.save(path, np.ascontiguousarray(embedding, dtype=np.float32))


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description="spectral_init on the GPU from a CSR .npz graph")
    p.add_argument("graph", type=Path)
    p.add_argument("out", type=Path)
    p.add_argument("--n-components", type=int, default=2)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--data", type=Path, default=None, help="points [n, d] (.npy), for graphs with many components")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    from . import api
    g = load_csr_npz(a.graph)
    data = np.load(a.data).astype(np.float32) if a.data is not None else None
    cfg = api.SpectralInitConfig(precision=api.Precision.MIXED if a.precision == "mixed" else api.Precision.FP64)
    emb, rep = api.spectral_init(g, a.n_components, a.seed, data=data, config=cfg,
                                 ctx=api.get_context(a.device), return_report=True)
    save_embedding(a.out, emb)
    print(f"n={g.shape[0]} nnz={g.nnz} components={rep.n_components_graph} level={rep.level} "
          f"iterations={rep.iterations} max_residual={rep.max_residual:.2e} -> {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
