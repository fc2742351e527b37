"""The fuzzy-kNN construction oracle (oracle/fuzzy_oracle.py) against the
reference's stage fixtures (tests/generate_fixtures.py:70-182): exact kNN,
smooth-kNN sigma / rho, membership strengths, fuzzy union, pruning.  Each
stage is fed the fixture's own inputs so that a failure points at one stage."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN
from oracle import fuzzy_oracle as F

DATASETS = ["blobs_connected_200", "moons_200", "near_dupes_100"]


def _npz(ds, name):
    return np.load(GOLDEN / ds / f"{name}.npz", allow_pickle=False)


def _csr(ds, name):
    return sp.load_npz(GOLDEN / ds / f"{name}.npz").tocsr()


@pytest.mark.parametrize("ds", DATASETS)
def test_knn_exact(ds):
    x = _npz(ds, "step0_raw_data")["X"]
    ref = _npz(ds, "step1_knn_exact")
    k = int(ref["n_neighbors"])
    idx, d = F.knn_exact(x, k)
    assert np.allclose(d, ref["knn_dists"], rtol=1e-6, atol=1e-7)
    if ds != "near_dupes_100":  # duplicated points tie; their order is not pinned
        assert np.array_equal(idx, ref["knn_indices"])


@pytest.mark.parametrize("ds", DATASETS)
def test_smooth_knn(ds):
    ref1 = _npz(ds, "step1_knn_exact")
    ref2 = _npz(ds, "step2_smooth_knn_exact")
    sig, rho = F.smooth_knn(ref1["knn_dists"], int(ref1["n_neighbors"]))
    assert np.allclose(rho, ref2["rhos"], rtol=0, atol=0)
    assert np.allclose(sig, ref2["sigmas"], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("ds", DATASETS)
def test_membership(ds):
    ref1 = _npz(ds, "step1_knn_exact")
    ref2 = _npz(ds, "step2_smooth_knn_exact")
    m = F.membership(ref1["knn_indices"], ref1["knn_dists"], ref2["sigmas"], ref2["rhos"]).tocsr()
    ref = _csr(ds, "step3_membership_exact")
    m.sort_indices()
    ref.sort_indices()
    assert np.array_equal(m.indptr, ref.indptr) and np.array_equal(m.indices, ref.indices)
    assert np.allclose(m.data, ref.data, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("ds", DATASETS)
def test_union_and_prune(ds):
    n = _npz(ds, "step0_raw_data")["X"].shape[0]
    u = F.fuzzy_union(_csr(ds, "step3_membership_exact"))
    ref4 = _csr(ds, "step4_symmetrized_exact")
    for a in (u, ref4):
        a.sort_indices()
    assert np.array_equal(u.indptr, ref4.indptr) and np.array_equal(u.indices, ref4.indices)
    assert np.allclose(u.data, ref4.data, rtol=1e-6, atol=1e-7)
    p = F.prune(ref4, n)
    ref5 = _csr(ds, "step5a_pruned_exact")
    p.sort_indices()
    ref5.sort_indices()
    assert np.array_equal(p.indptr, ref5.indptr) and np.array_equal(p.indices, ref5.indices)
    assert np.allclose(p.data, ref5.data, rtol=0, atol=0)
