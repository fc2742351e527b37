"""The CPU oracle pinned against the crate's golden fixtures (the same
tolerances as tests/integration/test_comp_*.rs of the reference)."""
import math
import struct

import numpy as np
import pytest

from conftest import ALL_DATASETS, CONNECTED, load_csr, load_graph, load_npz
from oracle import spectral_oracle as O


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_degrees_python_compat_bit_exact(ds):
    # test_comp_a_degrees.rs:41-60 (1e-15, bit-for-bit)
    g = load_graph(ds)
    deg, sq = O.compute_degrees(g, O.PYTHON_COMPAT)
    ref = load_npz(ds, "comp_a_degrees.npz")
    assert np.array_equal(deg, ref["degrees"])
    assert np.array_equal(sq, ref["sqrt_deg"])


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_degrees_rust_native(ds):
    # test_comp_a_degrees.rs:66-81 (3e-7 relative)
    g = load_graph(ds)
    deg, _ = O.compute_degrees_rust_native_fast(g)
    ref = load_npz(ds, "comp_a_degrees.npz")["degrees"]
    assert np.all(np.abs(deg - ref) < 3e-7 * np.maximum(np.abs(ref), 1.0))


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_laplacian_matches_golden(ds):
    # test_comp_b_laplacian.rs:29-53
    g = load_graph(ds)
    sq = load_npz(ds, "comp_a_degrees.npz")["sqrt_deg"]
    lap = O.build_normalized_laplacian(g, O.inv_sqrt(sq))
    ref = load_csr(ds, "comp_b_laplacian.npz")
    assert abs(lap - ref).max() < 1e-14 if lap.nnz else True
    assert abs(lap - lap.T).max() < 1e-15
    assert np.all(np.abs(lap.diagonal() - 1.0) < 1e-15)


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_components_match_golden(ds):
    g = load_graph(ds)
    lab, nc = O.find_components(g)
    ref = load_npz(ds, "comp_c_components.npz")
    assert nc == int(ref["n_components"])
    assert np.array_equal(lab, ref["labels"])
    lab2, nc2 = O.find_components_fast(g)
    assert nc2 == nc and np.array_equal(lab2, lab)


@pytest.mark.parametrize("ds", ["blobs_connected_200", "moons_200", "near_dupes_100", "circles_300"])
def test_dense_evd_matches_golden(ds):
    # test_comp_d_dense_evd.rs:28-60
    lap = load_csr(ds, "comp_b_laplacian.npz")
    ref = load_npz(ds, "comp_d_eigensolver.npz")
    vals, vecs = O.dense_evd(lap, len(ref["eigenvalues"]))
    assert np.all(np.abs(vals - ref["eigenvalues"]) < 1e-9)
    for j in range(len(vals)):
        assert O.eigenpair_residual(lap, vecs[:, j], vals[j]) < 1e-10


@pytest.mark.parametrize("ds", CONNECTED)
@pytest.mark.parametrize("regularize", [False, True])
def test_lobpcg_oracle_matches_golden(ds, regularize):
    # test_comp_f_lobpcg.rs:22-62
    lap = load_csr(ds, "comp_b_laplacian.npz")
    sq = load_npz(ds, "comp_a_degrees.npz")["sqrt_deg"]
    r = O.lobpcg_solve(O.CsrOperator(lap), 2, 42, regularize, sq)
    assert r is not None
    (vals, vecs), _ = r
    ref = load_npz(ds, "comp_d_eigensolver.npz")["eigenvalues"]
    if not regularize:
        assert np.all(np.abs(vals - ref) < 1e-6)
    for j in range(3):
        assert O.eigenpair_residual(lap, vecs[:, j], vals[j]) < 1e-5


@pytest.mark.parametrize("ds", ["blobs_connected_200", "blobs_connected_2000", "moons_200", "circles_300",
                                "near_dupes_100"])
def test_rsvd_oracle_sanity(ds):
    # test_comp_d_rsvd.rs:41-66 (sanity 5e-1)
    lap = load_csr(ds, "comp_b_laplacian.npz")
    ref = load_npz(ds, "comp_d_eigensolver.npz")["eigenvalues"]
    vals, vecs = O.rsvd_solve(lap, 2, 42)
    for i in range(2):
        assert abs(vals[i + 1] - ref[i + 1]) < 5e-1
        assert O.eigenpair_residual(lap, vecs[:, i + 1], vals[i + 1]) < 5e-1


@pytest.mark.parametrize("ds", ["blobs_connected_200", "moons_200", "circles_300", "near_dupes_100"])
def test_selection_matches_golden(ds):
    # test_comp_e_selection.rs:31-56
    d = load_npz(ds, "comp_d_eigensolver.npz")
    e = load_npz(ds, "comp_e_selection.npz")
    sel = O.select_eigenvectors(d["eigenvalues"], d["eigenvectors"], 2)
    for c in range(2):
        s = np.sign(sel[:, c] @ e["embedding"][:, c])
        assert np.max(np.abs(sel[:, c] - s * e["embedding"][:, c])) < 1e-10


@pytest.mark.parametrize("ds", CONNECTED)
def test_scaling_matches_golden(ds):
    # comp_f_scaling: pre_noise = embedding * expansion (f32); expansion = 10 / max|embedding|
    e = load_npz(ds, "comp_e_selection.npz")["embedding"]
    f = load_npz(ds, "comp_f_scaling.npz")
    scaled = O.scale_coords(e, 10.0)
    assert np.allclose(10.0 / np.max(np.abs(e)), float(f["expansion"]), rtol=1e-12)
    assert np.max(np.abs(scaled - f["pre_noise"])) <= 1e-5


@pytest.mark.parametrize("ds", CONNECTED)
def test_oracle_pipeline_residual(ds):
    # test_e2e_validation.rs:23-77: de-scaled output is an eigenvector pair (residual < 0.005)
    g = load_graph(ds)
    out = O.spectral_init(g, 2, 42)
    f = load_npz(ds, "comp_f_scaling.npz")
    lap = load_csr(ds, "comp_b_laplacian.npz")
    ref = load_npz(ds, "comp_d_eigensolver.npz")["eigenvalues"]
    des = out.astype(np.float64) / float(f["expansion"])
    for c in range(2):
        assert O.eigenpair_residual(lap, des[:, c], ref[c + 1]) < 0.005


def test_oracle_sign_convention():
    x = np.array([[1.0, -3.0], [-2.0, 3.0], [0.5, 1.0]])
    O.normalize_signs(x)
    assert x[1, 0] == 2.0 and x[0, 1] == 3.0  # first max-|.| entry made positive


def _rust_total_cmp_key(v: float) -> int:
    # f64::total_cmp: bits as i64, negative values with the magnitude bits flipped
    (b,) = struct.unpack("<q", struct.pack("<d", v))
    return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFF)


def _rust_column_sign(col) -> float:
    # src/scaling.rs:64-69: reduce(|a, b| if |b|.total_cmp(|a|).is_gt() { b } else { a }).signum()
    best = None
    for b in col:
        if best is None or _rust_total_cmp_key(abs(b)) > _rust_total_cmp_key(abs(best)):
            best = b
    if best is None:
        return 1.0
    if math.isnan(best):
        return math.nan
    return math.copysign(1.0, best)


def test_oracle_sign_rule_matches_total_cmp_reduce():
    nan_a = struct.unpack("<d", struct.pack("<Q", 0x7FF8000000000001))[0]
    nan_b = struct.unpack("<d", struct.pack("<Q", 0xFFF8000000000002))[0]  # larger payload, sign bit set
    cols = [
        [1.0, -3.0, 3.0, 0.5],            # tie +-3: the first (negative) wins -> flip
        [-0.0, 0.0, -0.0],                # all zeros: first (-0.0) -> signum -1 -> flip
        [-2.0, math.nan, -7.0],           # NaN ranks above every finite value -> never flipped
        [-math.inf, 5.0, -1.0],           # -inf is the maximum -> flip
        [-4.0, nan_a, nan_b, -9.0],       # NaNs rank by payload (|.| clears the sign bit)
        [0.25, -0.5, 0.5],
    ]
    rng = np.random.default_rng(3)
    cols += [list(rng.standard_normal(17)) for _ in range(5)]
    for col in cols:
        x = np.array(col, dtype=np.float64)[:, None].copy()
        O.normalize_signs(x)
        flipped = not (_rust_column_sign(col) >= 0.0 or math.isnan(_rust_column_sign(col)))
        expect = -np.array(col) if flipped else np.array(col)
        got = x[:, 0]
        same = (got.view(np.uint64) == expect.view(np.uint64)) | (np.isnan(got) & np.isnan(expect))
        assert same.all(), (col, got, expect)


def test_oracle_errors():
    import scipy.sparse as sp
    g = sp.csr_matrix((np.ones(4, np.float32), ([0, 1, 1, 2], [1, 0, 2, 1])), shape=(3, 3))
    with pytest.raises(O.InvalidGraph):
        O.spectral_init(g, 0, 42)
    with pytest.raises(O.TooFewNodes):
        O.spectral_init(sp.csr_matrix((np.ones(2, np.float32), ([0, 1], [1, 0])), shape=(2, 2)), 3, 42)
    with pytest.raises(O.InvalidGraph):
        O.spectral_init(sp.csr_matrix((0, 0), dtype=np.float32), 2, 42)
