"""Device eigensolvers vs the golden fixtures and the reference's own unit
tests (src/solvers/lobpcg.rs:499-883, dense.rs:78-149, rsvd.rs tests,
tests/integration/test_comp_{d,f}_*.rs)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import CONNECTED, load_csr, load_npz
from oracle import spectral_oracle as O

pytestmark = pytest.mark.gpu


def diagonal_csr(values):
    n = len(values)
    return sp.csr_matrix((np.asarray(values, dtype=np.float64), np.arange(n), np.arange(n + 1)), shape=(n, n))


def resid(mat, v, lam):
    return O.eigenpair_residual(mat, v, lam)


# ---- dense EVD ---------------------------------------------------------------------------------
@pytest.mark.parametrize("ds", ["blobs_connected_200", "moons_200", "near_dupes_100", "circles_300"])
def test_dense_evd_matches_golden(gpu_ctx, ds):
    import spectral_init_b200 as si
    lap = load_csr(ds, "comp_b_laplacian.npz")
    ref = load_npz(ds, "comp_d_eigensolver.npz")
    k = len(ref["eigenvalues"])
    vals, vecs = si.dense_evd(lap, k, ctx=gpu_ctx)
    assert np.all(np.abs(vals - ref["eigenvalues"]) < 1e-9)
    for j in range(k):
        assert resid(lap, vecs[:, j], vals[j]) < 1e-10
    gaps = ref["eigenvalue_gaps"]
    for j in range(len(gaps)):
        if gaps[j] < 1e-6:
            g = vecs[:, j:j + 2].T @ ref["eigenvectors"][:, j:j + 2]
            assert abs(np.linalg.det(g)) > 0.99


def test_dense_evd_known_answers(gpu_ctx):
    import spectral_init_b200 as si
    # [[1,-1],[-1,1]] -> 0, 2 (src/solvers/dense.rs:78-)
    m = sp.csr_matrix(np.array([[1.0, -1.0], [-1.0, 1.0]]))
    vals, vecs = si.dense_evd(m, 2, ctx=gpu_ctx)
    assert np.allclose(vals, [0.0, 2.0], atol=1e-12)
    # path Laplacian spectrum 2 - 2 cos(pi j / n)
    n = 40
    p = sp.diags([-np.ones(n - 1), np.r_[1.0, 2 * np.ones(n - 2), 1.0], -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    vals, vecs = si.dense_evd(p, 5, ctx=gpu_ctx)
    want = 2 - 2 * np.cos(np.pi * np.arange(5) / n)
    assert np.allclose(vals, want, atol=1e-12)
    # block diagonal with a repeated zero eigenvalue: any orthonormal basis, residual tiny
    b = sp.block_diag([p, p, p]).tocsr()
    vals, vecs = si.dense_evd(b, 4, ctx=gpu_ctx)
    assert np.allclose(vals[:3], 0.0, atol=1e-12)
    assert np.allclose(vecs.T @ vecs, np.eye(4), atol=1e-10)
    for j in range(4):
        assert resid(b, vecs[:, j], vals[j]) < 1e-10
    with pytest.raises(si.TooFewNodes):
        si.dense_evd(m, 3, ctx=gpu_ctx)


# ---- LOBPCG -----------------------------------------------------------------------------------
@pytest.mark.parametrize("ds", CONNECTED)
@pytest.mark.parametrize("regularize", [False, True])
def test_lobpcg_matches_golden(gpu_ctx, ds, regularize):
    import spectral_init_b200 as si
    lap = load_csr(ds, "comp_b_laplacian.npz")
    sq = load_npz(ds, "comp_a_degrees.npz")["sqrt_deg"]
    r = si.lobpcg_solve(lap, 2, 42, regularize, sq, ctx=gpu_ctx)
    assert r is not None
    (vals, vecs), _ = r
    ref = load_npz(ds, "comp_d_eigensolver.npz")["eigenvalues"]
    if not regularize:
        assert np.all(np.abs(vals - ref) < 1e-6), (vals, ref)
    for j in range(3):
        assert resid(lap, vecs[:, j], vals[j]) < 1e-5


def test_lobpcg_injects_trivial_eigenvector(gpu_ctx):
    import spectral_init_b200 as si
    n = 20
    diag = [1e-10] + [i * 0.1 for i in range(1, n)]
    mat = diagonal_csr(diag)
    r = si.lobpcg_solve(mat, 2, 42, False, np.sqrt(diag), ctx=gpu_ctx)
    assert r is not None
    (vals, vecs), _ = r
    assert vals[0] < 1e-6
    for i in range(3):
        assert resid(mat, vecs[:, i], vals[i]) < 1e-5


@pytest.mark.parametrize("regularize", [False, True])
def test_lobpcg_diagonal(gpu_ctx, regularize):
    import spectral_init_b200 as si
    diag = [0.0, 0.1, 0.3, 0.7, 1.2, 2.0]
    mat = diagonal_csr(diag)
    r = si.lobpcg_solve(mat, 2, 42, regularize, np.ones(6), ctx=gpu_ctx)
    assert r is not None
    (vals, vecs), _ = r
    assert abs(vals[0] - 0.0) < 1e-6 and abs(vals[1] - 0.1) < 1e-6
    for i in range(3):
        assert resid(mat, vecs[:, i], vals[i]) < 1e-5


def test_lobpcg_returns_k_plus_one_and_orthonormal(gpu_ctx):
    import spectral_init_b200 as si
    mat = diagonal_csr(np.arange(1, 31, dtype=float))
    (vals, vecs), _ = si.lobpcg_solve(mat, 3, 42, False, np.ones(30), ctx=gpu_ctx)
    assert vals.shape == (4,) and vecs.shape == (30, 4)
    mat = diagonal_csr(np.arange(1, 9) * 0.25)
    (vals, vecs), _ = si.lobpcg_solve(mat, 3, 42, False, np.ones(8), ctx=gpu_ctx)
    assert np.allclose(vals, [0.25, 0.5, 0.75, 1.0], atol=1e-6)
    assert np.allclose(vecs.T @ vecs, np.eye(4), atol=1e-8)
    for i in range(4):
        assert resid(mat, vecs[:, i], vals[i]) < 1e-8


def test_lobpcg_near_degenerate_n2000(gpu_ctx):
    import spectral_init_b200 as si
    n = 2000
    diag = [1e-4, 2e-4] + [0.1 + (i - 2.0) * 0.1 / (n - 2.0) for i in range(2, n)]
    mat = diagonal_csr(diag)
    r = si.lobpcg_solve(mat, 2, 42, False, np.ones(n), ctx=gpu_ctx)
    assert r is not None
    (vals, vecs), _ = r
    for i in range(3):
        assert resid(mat, vecs[:, i], vals[i]) < 1e-5


def test_lobpcg_restart_count_zero_on_uniform_diagonal(gpu_ctx):
    import spectral_init_b200 as si
    mat = diagonal_csr(np.ones(8))
    r = si.lobpcg_solve(mat, 2, 42, False, np.ones(8), ctx=gpu_ctx)
    assert r is not None and r[1] == 0


def test_lobpcg_precondition_failures_return_none(gpu_ctx):
    import spectral_init_b200 as si
    mat = diagonal_csr([0.0, 0.5, 1.0])
    assert si.lobpcg_solve(mat, 2, 42, False, np.ones(3), ctx=gpu_ctx) is None      # k >= n
    assert si.lobpcg_solve(mat, 0, 42, False, np.ones(3), ctx=gpu_ctx) is None      # n_components == 0
    assert si.lobpcg_solve(mat, 1, 42, False, np.ones(2), ctx=gpu_ctx) is None      # sqrt_deg length


# ---- rSVD ----------------------------------------------------------------------------------------
@pytest.mark.parametrize("ds", ["blobs_connected_200", "blobs_connected_2000", "moons_200", "circles_300",
                                "near_dupes_100"])
def test_rsvd_sanity(gpu_ctx, ds):
    """test_comp_d_rsvd.rs sanity tolerances (5e-1).  The crate's default width
    K = rank + max(n/10, rank, 5) (src/solvers/rsvd.rs:84-87) is honoured where
    it fits the device limit of 64 columns; above it the call is an explicit
    SI_INVALID_ARGUMENT naming the limit, and the widest allowed subspace runs."""
    import spectral_init_b200 as si
    from spectral_init_b200.api import InvalidArgument
    lap = load_csr(ds, "comp_b_laplacian.npz")
    ref = load_npz(ds, "comp_d_eigensolver.npz")["eigenvalues"]
    n = lap.shape[0]
    default_k = 3 + min(max(n // 10, 5), n - 3)
    over = None
    if default_k > 64:
        with pytest.raises(InvalidArgument, match="64"):
            si.rsvd_solve(lap, 2, 42, ctx=gpu_ctx)
        over = 64 - 3
    vals, vecs = si.rsvd_solve(lap, 2, 42, oversampling=over, ctx=gpu_ctx)
    for i in range(2):
        assert abs(vals[i + 1] - ref[i + 1]) < 5e-1
        assert resid(lap, vecs[:, i + 1], vals[i + 1]) < 5e-1


def test_rsvd_more_power_iterations_converge(gpu_ctx):
    import spectral_init_b200 as si
    lap = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    ref = load_npz("blobs_connected_2000", "comp_d_eigensolver.npz")["eigenvalues"]
    v2, _ = si.rsvd_solve(lap, 2, 42, oversampling=30, nbiter=2, ctx=gpu_ctx)
    v8, x8 = si.rsvd_solve(lap, 2, 42, oversampling=50, nbiter=8, ctx=gpu_ctx)
    assert abs(v8[1] - ref[1]) <= abs(v2[1] - ref[1]) + 1e-12
    assert resid(lap, x8[:, 1], v8[1]) < 5e-2


# ---- escalation chain ------------------------------------------------------------------------------
def test_chain_levels(gpu_ctx):
    import spectral_init_b200 as si
    small = load_csr("moons_200", "comp_b_laplacian.npz")
    (vals, vecs), level = si.solve_eigenproblem_pub(small, 2, 42, ctx=gpu_ctx)
    assert level == 0
    big = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    (vals, vecs), level = si.solve_eigenproblem_pub(big, 2, 42, ctx=gpu_ctx)
    assert level == 1
    assert O.max_eigenpair_residual(big, vals, vecs) < 1e-5
    ref = load_npz("blobs_connected_2000", "comp_d_eigensolver.npz")["eigenvalues"]
    assert np.all(np.abs(vals - ref) < 1e-6)


@pytest.mark.parametrize("level", [0, 1, 2, 3, 4, 5])
def test_forced_levels(gpu_ctx, level):
    import spectral_init_b200 as si
    lap = load_csr("circles_300", "comp_b_laplacian.npz")
    cfg = si.SpectralInitConfig(force_level=level)
    (vals, vecs), got = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx)
    assert got == level
    assert np.all(np.diff(vals) >= -1e-9)          # ascending (invariant B1)
    tol = {0: 1e-10, 1: 1e-5, 2: 1e-6, 3: 1e-5, 4: 5e-1, 5: 1e-10}[level]
    assert O.max_eigenpair_residual(lap, vals, vecs) < tol


@pytest.mark.parametrize("dataset", ["blobs_connected_2000", "moons_200", "near_dupes_100"])
def test_shift_invert_level_matches_golden(gpu_ctx, dataset):
    """Level 2 (src/solvers/sinv.rs:106-189): eigenvalues within 1e-6 of the golden
    ones and the 1e-6 residual gate of the crate (src/metrics.rs:35)."""
    import spectral_init_b200 as si
    lap = load_csr(dataset, "comp_b_laplacian.npz")
    ref = load_npz(dataset, "comp_d_eigensolver.npz")["eigenvalues"]
    cfg = si.SpectralInitConfig(force_level=2)
    (vals, vecs), got = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx)
    assert got == 2
    assert np.all(np.abs(vals - ref[:3]) < 1e-6), (vals, ref[:3])
    assert O.max_eigenpair_residual(lap, vals, vecs) < 1e-6


# ---- dense EVD: single-launch vs multi-launch tridiagonalisation --------------------------------
@pytest.mark.parametrize("n", [192, 517, 1999])
@pytest.mark.parametrize("path", ["coop", "steps"])
def test_dense_evd_tridiag_paths(gpu_ctx, monkeypatch, n, path):
    """Both tridiagonalisations (one cooperative launch with the matrix in the
    CTAs' shared memory; three launches per column) against LAPACK on a
    random weighted graph Laplacian and on a path graph with known spectrum."""
    import spectral_init_b200 as si
    if path == "steps":
        monkeypatch.setenv("SPECTRAL_INIT_TRIDIAG", "steps")
    rng = np.random.default_rng(n)
    # random sparse graph: a ring (connected) plus random chords, normalised Laplacian
    rows = np.r_[np.arange(n), rng.integers(0, n, 4 * n)]
    cols = np.r_[(np.arange(n) + 1) % n, rng.integers(0, n, 4 * n)]
    w = rng.uniform(0.1, 1.0, rows.size)
    a = sp.coo_matrix((w, (rows, cols)), shape=(n, n)).tocsr()
    a = a + a.T
    a.setdiag(0.0)
    a.eliminate_zeros()
    dinv = 1.0 / np.sqrt(np.asarray(a.sum(axis=1)).ravel())
    lap = (sp.identity(n) - sp.diags(dinv) @ a @ sp.diags(dinv)).tocsr()
    k = 6
    vals, vecs = si.dense_evd(lap, k, ctx=gpu_ctx)
    want = np.linalg.eigvalsh(lap.toarray())[:k]
    assert np.max(np.abs(vals - want)) < 1e-10
    assert np.allclose(vecs.T @ vecs, np.eye(k), atol=1e-10)
    for j in range(k):
        assert resid(lap, vecs[:, j], vals[j]) < 1e-10
    # path Laplacian: 2 - 2 cos(pi j / n)
    p = sp.diags([-np.ones(n - 1), np.r_[1.0, 2 * np.ones(n - 2), 1.0], -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    vals, vecs = si.dense_evd(p, 4, ctx=gpu_ctx)
    assert np.allclose(vals, 2 - 2 * np.cos(np.pi * np.arange(4) / n), atol=1e-11)
    for j in range(4):
        assert resid(p, vecs[:, j], vals[j]) < 1e-10


# ---- LOBPCG with 8- and 16-column blocks (register-tiled Gram, four-column update) -------------
@pytest.mark.parametrize("nc,block", [(5, 0), (5, 7), (8, 0), (8, 10), (12, 0)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lobpcg_wide_blocks(gpu_ctx, nc, block, precision):
    """LOBPCG whose blocks are padded to 8 or 16 columns (m = the padded width
    by default, m < width with an explicit block size) against LAPACK."""
    import spectral_init_b200 as si
    n = 1800
    rng = np.random.default_rng(nc * 100 + block)
    rows = np.r_[np.arange(n), rng.integers(0, n, 3 * n)]
    cols = np.r_[(np.arange(n) + 1) % n, rng.integers(0, n, 3 * n)]
    a = sp.coo_matrix((rng.uniform(0.1, 1.0, rows.size), (rows, cols)), shape=(n, n)).tocsr()
    a = a + a.T
    a.setdiag(0.0)
    a.eliminate_zeros()
    deg = np.asarray(a.sum(axis=1)).ravel()
    dinv = 1.0 / np.sqrt(deg)
    lap = (sp.identity(n) - sp.diags(dinv) @ a @ sp.diags(dinv)).tocsr()
    cfg = si.SpectralInitConfig(precision=si.Precision.MIXED if precision == "mixed" else si.Precision.FP64,
                                block_size=block)
    out = si.lobpcg_solve(lap, nc, 42, False, np.sqrt(deg), cfg, ctx=gpu_ctx)
    assert out is not None
    (vals, vecs), _ = out
    k = nc + 1
    want = np.linalg.eigvalsh(lap.toarray())[:k]
    # residual 1e-5 bounds the eigenvalue error by ~1e-10 / gap
    assert np.max(np.abs(vals - want)) < 1e-7
    assert np.allclose(vecs.T @ vecs, np.eye(k), atol=1e-8)
    for j in range(k):
        assert resid(lap, vecs[:, j], vals[j]) < 1e-5


@pytest.mark.parametrize("variant", ["task", "tile"])
@pytest.mark.parametrize("small", ["warp", "cta", "serial", "reg"])
def test_lobpcg_kernel_variants_agree(gpu_ctx, monkeypatch, variant, small):
    """The 4-column LOBPCG iteration with either Gram kernel (task-split warps,
    default; register-tiled, SPECTRAL_INIT_GRAM=tile) and each small step (one
    warp with the Gram in shared memory, SPECTRAL_INIT_SMALL_STEP=warp; one
    128-thread CTA with the parallel Rayleigh-Ritz, the default; the same CTA
    with one-thread-per-column triangular solves, =serial; one warp in
    registers, =reg) converges to the dense eigenpairs."""
    import spectral_init_b200 as si
    if variant == "tile":
        monkeypatch.setenv("SPECTRAL_INIT_GRAM", "tile")
    monkeypatch.setenv("SPECTRAL_INIT_SMALL_STEP", small)
    lap = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    cfg = si.SpectralInitConfig(force_level=1, tol=1e-10)
    (vals, vecs), level = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx)
    w = np.linalg.eigvalsh(lap.toarray())[:3]
    assert level == 1
    assert np.all(np.abs(vals - w) < 1e-10), (vals, w)
    assert O.max_eigenpair_residual(lap, vals, vecs) < 1e-9


@pytest.mark.parametrize("kernel", ["sell", "sell_pf_pipe", "panel", "vec4", "tiled4"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lobpcg_spmm_variants_agree(gpu_ctx, monkeypatch, kernel, precision):
    """The LOBPCG solve (with its fused SpMM epilogues and the mixed-precision
    f32 phase) with each SpMM kernel forced converges to the dense eigenpairs."""
    import spectral_init_b200 as si
    monkeypatch.setenv("SPECTRAL_INIT_SPMM_KERNEL", kernel)
    lap = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    prec = si.Precision.MIXED if precision == "mixed" else si.Precision.FP64
    cfg = si.SpectralInitConfig(force_level=1, tol=1e-10, precision=prec)
    (vals, vecs), level = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx)
    w = np.linalg.eigvalsh(lap.toarray())[:3]
    assert level == 1
    assert np.all(np.abs(vals - w) < 1e-10), (vals, w)
    assert O.max_eigenpair_residual(lap, vals, vecs) < 1e-9
