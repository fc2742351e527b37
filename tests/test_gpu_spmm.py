"""CSR SpMM (LinearOperator::apply) on the device vs scipy in f64."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_csr
from oracle import graphgen

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 8, 9, 16, 17])
def test_spmm_f64_matches_scipy_on_golden_laplacian(gpu_ctx, k):
    import torch
    import spectral_init_b200 as si
    lap = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    op = si.CsrOperator(lap, diag=0.0, ctx=gpu_ctx)
    rng = np.random.default_rng(k)
    x = rng.standard_normal((lap.shape[0], k))
    y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    assert _rel(y, lap @ x) < 1e-14


@pytest.mark.parametrize("deg_profile", ["sparse", "knn", "dense"])
@pytest.mark.parametrize("k", [4, 8, 16])
def test_spmm_vector_paths_all_group_widths(gpu_ctx, deg_profile, k):
    """Row lengths that select 4/8/16/32 lanes per row, with the implicit diagonal."""
    import torch
    import spectral_init_b200 as si
    n = 20000
    dens = {"sparse": 3.0, "knn": 16.0, "dense": 80.0}[deg_profile] / n
    a = sp.random(n, n, density=dens, random_state=1, format="csr")
    a = (a + a.T).tocsr()
    a.sort_indices()
    op = si.CsrOperator(a, diag=1.0, ctx=gpu_ctx)
    x = np.random.default_rng(0).standard_normal((n, k))
    y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    assert _rel(y, x + a @ x) < 1e-14


def test_spmm_f32_values_and_blocks(gpu_ctx):
    import torch
    import spectral_init_b200 as si
    g = graphgen.fuzzy_knn_graph(graphgen.gaussian_mixture(6000, 8, 10, seed=4), 15)
    _, sq = graphgen.degrees_f64(g)
    from oracle import spectral_oracle as O
    lap = O.build_normalized_laplacian(g, O.inv_sqrt(sq))
    op = si.CsrOperator(lap, diag=0.0, ctx=gpu_ctx, with_f32=True)
    x = np.random.default_rng(1).standard_normal((lap.shape[0], 4)).astype(np.float32)
    y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = lap @ x.astype(np.float64)
    # f32 values and blocks, f64 accumulation: error ~ a few f32 ulps of the row magnitude
    assert _rel(y, ref) < 2e-6


def test_spmm_empty_rows(gpu_ctx):
    import torch
    import spectral_init_b200 as si
    a = sp.csr_matrix((np.array([2.0, 3.0]), np.array([3, 0]), np.array([0, 1, 1, 1, 2, 2])), shape=(5, 5))
    op = si.CsrOperator(a, diag=0.5, ctx=gpu_ctx)
    x = np.arange(20, dtype=np.float64).reshape(5, 4)
    y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(y, 0.5 * x + a @ x)


_VARIANT_CACHE = {}


def _variant_matrix():
    """30 011 rows with ~32 entries per row (symmetrised), one empty row and one
    row longer than a staging block; built once per session."""
    if "a" not in _VARIANT_CACHE:
        rng = np.random.default_rng(7)
        n = 30_011
        nnz = 16 * n
        r = rng.integers(0, n, nnz)
        c = rng.integers(0, n, nnz)
        keep = (r != 5) & (c != 5)
        r, c = r[keep], c[keep]
        long_cols = rng.choice(n, 3000, replace=False)
        long_cols = long_cols[long_cols != 5]
        r = np.concatenate([r, np.full(long_cols.size, 17)])
        c = np.concatenate([c, long_cols])
        v = rng.uniform(0.1, 1.0, r.size)
        a = sp.csr_matrix((v, (r, c)), shape=(n, n))
        a = (a + a.T).tocsr()
        a.sum_duplicates()
        a.sort_indices()
        _VARIANT_CACHE["a"] = a
    return _VARIANT_CACHE["a"]


@pytest.mark.parametrize("kernel", ["vec4", "vec8", "vec16", "vec32", "tiled4", "tiled8", "gather4", "gather8",
                                    "panel"])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_spmm_every_kernel_variant(gpu_ctx, kernel, prec):
    """Each SpMM variant the autotuner can pick (SPECTRAL_INIT_SPMM_KERNEL forces
    one; the TMA gather4 variants apply to f32 values with 4-wide f32 blocks,
    f64 falls back to the tuned kernel), with an empty row, a long row and the
    implicit diagonal, against scipy in f64."""
    import os
    import torch
    import spectral_init_b200 as si
    a = _variant_matrix()
    n = a.shape[0]
    op = si.CsrOperator(a, diag=1.0, ctx=gpu_ctx, with_f32=(prec == "f32"))
    dt = np.float32 if prec == "f32" else np.float64
    x = np.random.default_rng(8).standard_normal((n, 4)).astype(dt)
    old = os.environ.get("SPECTRAL_INIT_SPMM_KERNEL")
    os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = kernel
    try:
        y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    finally:
        if old is None:
            del os.environ["SPECTRAL_INIT_SPMM_KERNEL"]
        else:
            os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = old
    vals = a.data.astype(np.float32).astype(np.float64) if prec == "f32" else a.data
    av = sp.csr_matrix((vals, a.indices, a.indptr), shape=a.shape)
    ref = x.astype(np.float64) + av @ x.astype(np.float64)
    assert _rel(y, ref) < (2e-6 if prec == "f32" else 1e-14)


def _clustered_matrix():
    """120 000 rows in 10 contiguous clusters of 12 000 (about 20 entries per
    row inside the cluster, 1 % of entries anywhere), symmetrised: the shape
    of a kNN graph of clustered points in cluster order."""
    if "c" not in _VARIANT_CACHE:
        rng = np.random.default_rng(11)
        n, size = 120_000, 12_000
        r = np.repeat(np.arange(n), 10)
        base = (r // size) * size
        c = base + rng.integers(0, size, r.size)
        far = rng.random(r.size) < 0.01
        c[far] = rng.integers(0, n, int(far.sum()))
        a = sp.csr_matrix((rng.uniform(0.1, 1.0, r.size), (r, c)), shape=(n, n))
        a = (a + a.T).tocsr()
        a.sum_duplicates()
        a.sort_indices()
        _VARIANT_CACHE["c"] = a
    return _VARIANT_CACHE["c"]


@pytest.mark.parametrize("width", [4, 8, 16])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_spmm_panel_windows_clustered(gpu_ctx, width, prec):
    """The panel kernel (x windows staged in shared memory, out-of-window
    entries gathered from global memory) on a cluster-ordered matrix larger
    than every window, for 4-, 8- and 16-wide blocks, against scipy in f64."""
    import os
    import torch
    import spectral_init_b200 as si
    a = _clustered_matrix()
    n = a.shape[0]
    op = si.CsrOperator(a, diag=1.0, ctx=gpu_ctx, with_f32=(prec == "f32"))
    dt = np.float32 if prec == "f32" else np.float64
    x = np.random.default_rng(9).standard_normal((n, width)).astype(dt)
    old = os.environ.get("SPECTRAL_INIT_SPMM_KERNEL")
    os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = "panel"
    try:
        y = op.apply(torch.from_numpy(x).cuda()).cpu().numpy()
    finally:
        if old is None:
            del os.environ["SPECTRAL_INIT_SPMM_KERNEL"]
        else:
            os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = old
    vals = a.data.astype(np.float32).astype(np.float64) if prec == "f32" else a.data
    av = sp.csr_matrix((vals, a.indices, a.indptr), shape=a.shape)
    ref = x.astype(np.float64) + av @ x.astype(np.float64)
    assert _rel(y, ref) < (2e-6 if prec == "f32" else 1e-14)


@pytest.mark.parametrize("width", [4, 8, 16])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_spmm_prepared_operator(gpu_ctx, width, prec):
    """si_spmm_planned (the prepared operator: partitions and panel windows
    built once) equals the one-shot si_spmm bit for bit and scipy to the
    kernels' tolerance, over repeated calls."""
    import torch
    import spectral_init_b200 as si
    a = _clustered_matrix()
    n = a.shape[0]
    op = si.CsrOperator(a, diag=1.0, ctx=gpu_ctx, with_f32=(prec == "f32"))
    dt = np.float32 if prec == "f32" else np.float64
    x = torch.from_numpy(np.random.default_rng(12).standard_normal((n, width)).astype(dt)).cuda()
    ref_once = op.apply(x)
    first = op.apply_prepared(x)
    gpu_ctx.synchronize()  # the planned call is queued on the library's stream
    first = first.clone()
    y = None
    for _ in range(3):
        y = op.apply_prepared(x, y)
    gpu_ctx.synchronize()
    # repeated planned calls are deterministic; the plan may pick the sliced
    # kernel (another summation order than the one-shot call), so the one-shot
    # result agrees to rounding
    assert torch.equal(y, first)
    tol = 2e-6 if prec == "f32" else 1e-14
    assert _rel(y.cpu().numpy().astype(np.float64), ref_once.cpu().numpy().astype(np.float64)) < tol
    vals = a.data.astype(np.float32).astype(np.float64) if prec == "f32" else a.data
    av = sp.csr_matrix((vals, a.indices, a.indptr), shape=a.shape)
    xh = x.cpu().numpy().astype(np.float64)
    assert _rel(y.cpu().numpy(), xh + av @ xh) < tol
    op.close()


@pytest.mark.parametrize("kernel", ["sell", "sell_pf", "sell_pipe", "sell_pf_pipe"])
@pytest.mark.parametrize("matrix", ["variant", "clustered"])
@pytest.mark.parametrize("width", [4, 8, 16])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_spmm_sliced_variants(gpu_ctx, kernel, matrix, width, prec):
    """The sliced-ELL kernels (one lane a row of a 32-row slice; rows sorted by
    length inside 256-row windows), forced through the prepared operator, on
    the random matrix with an empty row and a 3000-entry row and on the
    cluster-ordered matrix, 4/8/16-wide blocks, against scipy in f64 and
    deterministic over repeated calls."""
    import os
    import torch
    import spectral_init_b200 as si
    a = _variant_matrix() if matrix == "variant" else _clustered_matrix()
    n = a.shape[0]
    dt = np.float32 if prec == "f32" else np.float64
    x = torch.from_numpy(np.random.default_rng(13).standard_normal((n, width)).astype(dt)).cuda()
    old = os.environ.get("SPECTRAL_INIT_SPMM_KERNEL")
    os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = kernel
    try:
        op = si.CsrOperator(a, diag=0.75, ctx=gpu_ctx, with_f32=(prec == "f32"))
        y1 = op.apply_prepared(x)
        gpu_ctx.synchronize()  # the planned call is queued on the library's stream
        y1 = y1.clone()
        y2 = op.apply_prepared(x)
        gpu_ctx.synchronize()
    finally:
        if old is None:
            del os.environ["SPECTRAL_INIT_SPMM_KERNEL"]
        else:
            os.environ["SPECTRAL_INIT_SPMM_KERNEL"] = old
    assert torch.equal(y1, y2)
    vals = a.data.astype(np.float32).astype(np.float64) if prec == "f32" else a.data
    av = sp.csr_matrix((vals, a.indices, a.indptr), shape=a.shape)
    xh = x.cpu().numpy().astype(np.float64)
    assert _rel(y1.cpu().numpy(), 0.75 * xh + av @ xh) < (2e-6 if prec == "f32" else 1e-14)
    op.close()


def test_spmm_tuning_file(gpu_ctx, monkeypatch, tmp_path):
    """SPECTRAL_INIT_SPMM_TUNE_FILE: the autotuner appends the choice it timed,
    keyed by the operator's shape (n, nnz, width, value and block types);
    operators of at least 2^22 stored entries are timed."""
    import torch
    import spectral_init_b200 as si
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("SPECTRAL_INIT_SPMM_TUNE_FILE", str(path))
    monkeypatch.delenv("SPECTRAL_INIT_SPMM_KERNEL", raising=False)
    rng = np.random.default_rng(21)
    n = 262_147  # a shape no other test uses, with enough entries (~4.7 M) to be timed
    a = sp.random(n, n, density=9.0 / n, random_state=rng, format="csr")
    a = (a + a.T).tocsr()
    a.sort_indices()
    op = si.CsrOperator(a, diag=1.0, ctx=gpu_ctx)
    x = torch.from_numpy(rng.standard_normal((n, 4))).cuda()
    y = op.apply_prepared(x)
    gpu_ctx.synchronize()
    xh = x.cpu().numpy()
    assert _rel(y.cpu().numpy(), xh + a @ xh) < 1e-14
    lines = [l.split() for l in path.read_text().splitlines()]
    mine = [l for l in lines if int(l[0]) == n and int(l[1]) == a.nnz]
    assert mine and all(len(l) == 9 and int(l[2]) == 4 and int(l[3]) == 8 and int(l[4]) == 8 for l in mine)
    op.close()
