"""Device graph preparation vs the oracle and the golden fixtures:
degrees (bit-exact), Laplacian (explicit CSR and implicit values), components."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ALL_DATASETS, load_csr, load_graph, load_npz
from oracle import spectral_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_degrees_python_compat_bit_exact(gpu_ctx, ds):
    import spectral_init_b200 as si
    g = load_graph(ds)
    deg, sq = si.compute_degrees(g, si.ComputeMode.PythonCompat, ctx=gpu_ctx)
    ref = load_npz(ds, "comp_a_degrees.npz")
    assert np.array_equal(deg, ref["degrees"])
    assert np.array_equal(sq, ref["sqrt_deg"])


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_degrees_rust_native_matches_oracle(gpu_ctx, ds):
    import spectral_init_b200 as si
    g = load_graph(ds)
    deg, sq = si.compute_degrees(g, si.ComputeMode.RustNative, ctx=gpu_ctx)
    odeg, osq = O.compute_degrees(g, O.RUST_NATIVE)
    assert np.array_equal(deg, odeg) and np.array_equal(sq, osq)
    ref = load_npz(ds, "comp_a_degrees.npz")["degrees"]
    assert np.all(np.abs(deg - ref) < 3e-7 * np.maximum(np.abs(ref), 1.0))


def test_degrees_non_symmetric_graph_matches_column_scatter(gpu_ctx):
    import spectral_init_b200 as si
    rng = np.random.default_rng(3)
    n = 3000
    a = sp.random(n, n, density=0.004, random_state=7, format="csr", dtype=np.float32)
    a.data = rng.random(a.nnz).astype(np.float32)
    a.sort_indices()
    deg, sq = si.compute_degrees(a, si.ComputeMode.PythonCompat, ctx=gpu_ctx)
    odeg, osq = O.compute_degrees(a, O.PYTHON_COMPAT)
    assert np.array_equal(deg, odeg) and np.array_equal(sq, osq)


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_laplacian_csr_matches_golden_and_oracle(gpu_ctx, ds):
    import spectral_init_b200 as si
    g = load_graph(ds)
    sq = load_npz(ds, "comp_a_degrees.npz")["sqrt_deg"]
    inv = O.inv_sqrt(sq)
    lap = si.build_normalized_laplacian(g, inv, ctx=gpu_ctx)
    ref = load_csr(ds, "comp_b_laplacian.npz")
    olap = O.build_normalized_laplacian(g, inv)
    assert lap.nnz == olap.nnz
    assert np.array_equal(lap.indptr, olap.indptr) and np.array_equal(lap.indices, olap.indices)
    assert np.array_equal(lap.data, olap.data)            # bit-exact with the crate's expression
    assert abs(lap - ref).max() < 1e-14
    assert np.all(lap.diagonal() == 1.0)


@pytest.mark.parametrize("ds", ["blobs_connected_2000", "circles_300", "blobs_5000"])
def test_laplacian_implicit_values(gpu_ctx, ds):
    import spectral_init_b200 as si
    g = load_graph(ds)
    inv = O.inv_sqrt(load_npz(ds, "comp_a_degrees.npz")["sqrt_deg"])
    v64, v32 = si.build_laplacian_values(g, inv, ctx=gpu_ctx, with_f32=True)
    coo = g.tocoo()
    want = np.where(coo.row == coo.col, 0.0, (-inv[coo.row]) * coo.data.astype(np.float64) * inv[coo.col])
    assert np.array_equal(v64, want)
    assert np.array_equal(v32, want.astype(np.float32))


def test_self_loops_dropped_and_diagonal_inserted(gpu_ctx):
    import spectral_init_b200 as si
    # path 0-1-2 with a self loop on node 1
    g = sp.csr_matrix((np.array([1, 1, 0.5, 1, 1], np.float32), np.array([1, 0, 1, 2, 1]), np.array([0, 1, 4, 5])),
                      shape=(3, 3))
    deg, sq = si.compute_degrees(g, ctx=gpu_ctx)
    odeg, osq = O.compute_degrees(g)
    assert np.array_equal(deg, odeg)
    lap = si.build_normalized_laplacian(g, O.inv_sqrt(sq), ctx=gpu_ctx)
    olap = O.build_normalized_laplacian(g, O.inv_sqrt(osq))
    assert np.array_equal(lap.toarray(), olap.toarray())


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_components_match_golden(gpu_ctx, ds):
    import spectral_init_b200 as si
    g = load_graph(ds)
    lab, nc = si.find_components(g, ctx=gpu_ctx)
    ref = load_npz(ds, "comp_c_components.npz")
    assert nc == int(ref["n_components"])
    assert np.array_equal(lab, ref["labels"])


def test_components_many_random_pieces(gpu_ctx):
    import spectral_init_b200 as si
    rng = np.random.default_rng(11)
    n = 50_000
    a = sp.random(n, n, density=1.5 / n, random_state=5, format="csr", dtype=np.float32)
    a = ((a + a.T) > 0).astype(np.float32).tocsr()
    a.sort_indices()
    lab, nc = si.find_components(a, ctx=gpu_ctx)
    olab, onc = O.find_components_fast(a)
    assert nc == onc and np.array_equal(lab, olab)
    assert nc > 100


@pytest.mark.parametrize("bad", ["range", "order", "indptr", "nan"])
def test_invalid_graphs_are_rejected(gpu_ctx, bad):
    import spectral_init_b200 as si
    indptr = np.array([0, 1, 3, 4], np.uint64)
    indices = np.array([1, 0, 2, 1], np.uint32)
    data = np.ones(4, np.float32)
    if bad == "range":
        indices[1] = 7
    elif bad == "order":
        indices[1], indices[2] = 2, 0
    elif bad == "indptr":
        indptr[3] = 9
    else:
        data[0] = np.nan
    with pytest.raises(si.InvalidGraph):
        si.spectral_init((indptr, indices, data, 3), 1, 42, ctx=gpu_ctx)
