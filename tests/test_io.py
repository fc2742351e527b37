"""CSR .npz input (the format of the reference's fixtures and loader,
tests/common/mod.rs:30-80) and embedding output, on the CPU."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import ALL_DATASETS, GOLDEN
from spectral_init_b200 import io as sio
from spectral_init_b200.api import InvalidGraph


@pytest.mark.parametrize("ds", ALL_DATASETS)
def test_load_golden_graph_matches_scipy(ds):
    path = GOLDEN / ds / "step5a_pruned.npz"
    g = sio.load_csr_npz(path)
    ref = sp.load_npz(path).tocsr()
    ref.sort_indices()
    assert g.dtype == np.float32 and g.shape == ref.shape
    assert np.array_equal(g.indptr, ref.indptr) and np.array_equal(g.indices, ref.indices)
    assert np.array_equal(g.data, ref.data.astype(np.float32))


def test_load_laplacian_as_f64():
    lap = sio.load_csr_npz(GOLDEN / "blobs_50" / "comp_b_laplacian.npz", value_dtype=np.float64)
    ref = sp.load_npz(GOLDEN / "blobs_50" / "comp_b_laplacian.npz")
    assert lap.dtype == np.float64 and abs(lap - ref).max() == 0.0


def test_round_trip_and_int64_indices(tmp_path):
    g = sio.load_csr_npz(GOLDEN / "moons_200" / "step5a_pruned.npz")
    p = tmp_path / "g.npz"
    sio.save_csr_npz(p, g)
    assert (sio.load_csr_npz(p) != g).nnz == 0
    assert (sp.load_npz(p).astype(np.float32) != g).nnz == 0  # scipy reads what we write
    np.savez(tmp_path / "g64.npz", data=g.data.astype(np.float64), indices=g.indices.astype(np.int64),
             indptr=g.indptr.astype(np.int64), format=np.array(b"csr"), shape=np.array(g.shape))
    assert (sio.load_csr_npz(tmp_path / "g64.npz") != g).nnz == 0


def test_unsorted_columns_are_sorted(tmp_path):
    np.savez(tmp_path / "u.npz", data=np.array([1.0, 2.0], np.float32), indices=np.array([2, 0], np.int32),
             indptr=np.array([0, 2, 2, 2], np.int32), format=np.array(b"csr"), shape=np.array([3, 3]))
    g = sio.load_csr_npz(tmp_path / "u.npz")
    assert list(g.indices) == [0, 2] and list(g.data) == [2.0, 1.0]


@pytest.mark.parametrize("bad", ["format", "shape", "indptr", "index"])
def test_malformed_files_raise_invalid_graph(tmp_path, bad):
    arrays = dict(data=np.ones(2, np.float32), indices=np.array([1, 0], np.int32),
                  indptr=np.array([0, 1, 2], np.int32), format=np.array(b"csr"), shape=np.array([2, 2]))
    if bad == "format":
        arrays["format"] = np.array(b"coo")
    elif bad == "shape":
        arrays["shape"] = np.array([2, 3])
    elif bad == "indptr":
        arrays["indptr"] = np.array([0, 2, 1], np.int32)
    else:
        arrays["indices"] = np.array([1, 5], np.int32)
    np.savez(tmp_path / "b.npz", **arrays)
    with pytest.raises(InvalidGraph):
        sio.load_csr_npz(tmp_path / "b.npz")


def test_save_embedding(tmp_path):
    e = np.arange(6, dtype=np.float64).reshape(3, 2)
    sio.save_embedding(tmp_path / "e.npy", e)
    got = np.load(tmp_path / "e.npy")
    assert got.dtype == np.float32 and np.array_equal(got, e.astype(np.float32))


@pytest.mark.gpu
def test_cli_embeds_npz_graph_on_gpu(gpu_ctx, tmp_path):
    """python -m spectral_init_b200.io graph.npz out.npy: the file path gives
    the same embedding as the in-memory call (same seed, same device)."""
    import spectral_init_b200 as si
    src = GOLDEN / "blobs_connected_200" / "step5a_pruned.npz"
    out = tmp_path / "emb.npy"
    assert sio.main([str(src), str(out), "--n-components", "2", "--seed", "42"]) == 0
    emb = np.load(out)
    ref = si.spectral_init(sio.load_csr_npz(src), 2, 42, ctx=gpu_ctx)
    assert emb.shape == (200, 2) and np.array_equal(emb, ref)
