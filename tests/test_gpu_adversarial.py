"""Adversarial graphs, solver invariants and failure paths on the device.

The graphs and assertions follow the reference's own suites
(tests/integration/test_adversarial_graphs.rs:395-652: barbell, path, star,
epsilon-bridge, K_{m,n}, ring, exponentially weighted path, single edge, K_n,
lollipop; tests/integration/test_solver_invariants.rs:57-269: invariants
B1-B8), with the graph builders written here in numpy.  On top of the
reference's checks, every Laplacian's eigenpairs are compared with the dense
FP64 oracle (eigenvalues within 1e-8 relative, eigenvectors within 1e-5 per
degenerate group).

Failure paths are driven from the host, never by a fault: an iteration cap
that makes level 1 fail so the chain escalates (src/solvers/mod.rs:70-224),
a cap on the learned-start pass so the solver falls back to the random start,
and a zero wait limit for the single-launch tridiagonalisation so that its
bounded waits run out and the multi-launch steps redo the matrix.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import certified as CERT
from oracle import spectral_oracle as O

pytestmark = pytest.mark.gpu


# ---- graph builders (f32 weights, sorted CSR) ----------------------------------------------
def _sym(n, edges):
    r = [a for a, _, _ in edges] + [b for _, b, _ in edges]
    c = [b for _, b, _ in edges] + [a for a, _, _ in edges]
    w = [x for _, _, x in edges] * 2
    g = sp.csr_matrix((np.asarray(w, np.float32), (np.asarray(r), np.asarray(c))), shape=(n, n))
    g.sum_duplicates()
    g.sort_indices()
    return g


def complete(n):
    return _sym(n, [(i, j, 1.0) for i in range(n) for j in range(i + 1, n)])


def eps_bridge(cs, bridge):
    e = [(i, j, 1.0) for i in range(cs) for j in range(i + 1, cs)]
    e += [(cs + i, cs + j, 1.0) for i in range(cs) for j in range(i + 1, cs)]
    e.append((cs - 1, cs, bridge))
    return _sym(2 * cs, e)


def star(n):
    return _sym(n, [(0, i, 1.0) for i in range(1, n)])


def bipartite(m, n):
    return _sym(m + n, [(i, m + j, 1.0) for i in range(m) for j in range(n)])


def path(n):
    return _sym(n, [(i, i + 1, 1.0) for i in range(n - 1)])


def ring(n):
    return _sym(n, [(i, (i + 1) % n, 1.0) for i in range(n)])


def exp_path(n):
    # edge i -- i+1 weighs 10^(-8 i / (n - 1)) in f32
    w = [float(np.float32(10.0) ** np.float32(-8.0 * i / (n - 1))) for i in range(n - 1)]
    return _sym(n, [(i, i + 1, w[i]) for i in range(n - 1)])


def lollipop(cs, pl):
    e = [(i, j, 1.0) for i in range(cs) for j in range(i + 1, cs)]
    e += [(i, i + 1, 1.0) for i in range(cs - 1, cs + pl - 1)]
    return _sym(cs + pl, e)


GRAPHS = {
    "barbell_20": lambda: eps_bridge(20, 1.0),
    "path_100": lambda: path(100),
    "star_50": lambda: star(50),
    "eps_bridge_20": lambda: eps_bridge(20, 1e-6),
    "bipartite_10_10": lambda: bipartite(10, 10),
    "ring_100": lambda: ring(100),
    "exp_path_100": lambda: exp_path(100),
    "complete_20": lambda: complete(20),
    "lollipop_10_20": lambda: lollipop(10, 20),
}


def _laplacian(g):
    _, sq = O.compute_degrees(g, O.PYTHON_COMPAT)
    return O.build_normalized_laplacian(g, O.inv_sqrt(sq)), sq


# ---- group 1: valid embeddings, plus the eigenpairs against the dense oracle -----------------
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_adversarial_valid_embedding(gpu_ctx, name):
    import spectral_init_b200 as si
    g = GRAPHS[name]()
    out = si.spectral_init(g, 2, 42, ctx=gpu_ctx)
    assert out.shape == (g.shape[0], 2) and np.all(np.isfinite(out))


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_adversarial_eigenpairs_vs_dense_oracle(gpu_ctx, name):
    """solve_eigenproblem on the graph's Laplacian (level 0 at these sizes)
    against LAPACK: eigenvalues within 1e-8 relative (1e-10 absolute near
    zero), eigenvectors within 1e-5 per degenerate group."""
    import spectral_init_b200 as si
    lap, _ = _laplacian(GRAPHS[name]())
    (vals, vecs), level = si.solve_eigenproblem_pub(lap, 2, 42, ctx=gpu_ctx)
    assert level == 0
    ref = CERT.reference_eigenpairs(lap, lap.shape[0], extra=0)  # all pairs: degenerate groups stay whole
    cmp = CERT.compare(vals, vecs, ref, wanted=[0, 1, 2])
    for i in range(3):
        tol = 1e-8 * abs(ref.vals[i]) if abs(ref.vals[i]) > 1e-2 else 1e-10
        assert abs(vals[i] - ref.vals[i]) <= tol, (name, i, vals, ref.vals[:3])
    assert cmp["sin_theta_max"] < 1e-5, (name, cmp)


def test_single_edge_returns_too_few_nodes(gpu_ctx):
    import spectral_init_b200 as si
    with pytest.raises(si.TooFewNodes):
        si.spectral_init(path(2), 2, 42, ctx=gpu_ctx)


# ---- group 2 / 3: community separation and coordinate stability -----------------------------
def _intra_spread(col, idx):
    v = col[idx]
    return float(v.max() - v.min())


@pytest.mark.parametrize("bridge", [1.0, 1e-6])
def test_bridge_separates_communities(gpu_ctx, bridge):
    import spectral_init_b200 as si
    emb = si.spectral_init(eps_bridge(20, bridge), 2, 42, ctx=gpu_ctx)
    x = emb[:, 0]
    a, b = np.arange(20), np.arange(20, 40)
    gap = abs(float(x[a].mean() - x[b].mean()))
    assert gap > max(_intra_spread(x, a), _intra_spread(x, b)), (bridge, gap)


@pytest.mark.parametrize("name", ["star_50", "bipartite_10_10"])
def test_coordinate_stability(gpu_ctx, name):
    import spectral_init_b200 as si
    emb = si.spectral_init(GRAPHS[name](), 2, 42, ctx=gpu_ctx)
    assert float(np.max(np.abs(emb))) < 20.0


# ---- group 4: solver levels ------------------------------------------------------------------
def _diag_lap(n):
    return sp.csr_matrix((np.arange(n) / (n - 1), np.arange(n), np.arange(n + 1)), shape=(n, n))


def _path_lap(n):
    return _laplacian(path(n))[0]


def test_level0_for_small_n(gpu_ctx):
    import spectral_init_b200 as si
    _, level = si.solve_eigenproblem_pub(_path_lap(6), 2, 42, ctx=gpu_ctx)
    assert level == 0


def test_level1_for_large_well_conditioned(gpu_ctx):
    import spectral_init_b200 as si
    _, level = si.solve_eigenproblem_pub(_diag_lap(2001), 2, 42, ctx=gpu_ctx)
    assert level == 1


def test_regularized_lobpcg_valid(gpu_ctx):
    import spectral_init_b200 as si
    lap = _diag_lap(2001)
    assert si.lobpcg_solve(lap, 2, 42, False, np.ones(2001), ctx=gpu_ctx) is not None
    r = si.lobpcg_solve(lap, 2, 42, True, np.ones(2001), ctx=gpu_ctx)
    assert r is not None
    (vals, _), _ = r
    assert np.all(np.isfinite(vals)) and np.all(vals >= -1e-6)


def test_rsvd_valid_on_large_path(gpu_ctx):
    """rSVD on P_2001 (the reference calls it with its default width; the
    device limit is 64 columns, so the widest allowed subspace is used)."""
    import spectral_init_b200 as si
    vals, vecs = si.rsvd_solve(_path_lap(2001), 2, 42, oversampling=61, ctx=gpu_ctx)
    assert len(vals) == 3 and np.all(vals >= -1e-3) and np.all(np.isfinite(vecs)) and abs(vals[0]) < 0.1


# ---- invariants B1-B8 (test_solver_invariants.rs) --------------------------------------------
def test_b1_eigenvalues_ascending(gpu_ctx):
    import spectral_init_b200 as si
    from conftest import load_csr
    (vals, _), _ = si.solve_eigenproblem_pub(load_csr("blobs_50", "comp_b_laplacian.npz"), 2, 42, ctx=gpu_ctx)
    assert np.all(vals[:-1] <= vals[1:] + 1e-12)


def test_b2_dense_threshold_routing(gpu_ctx):
    """The crate's SPECTRAL_DENSE_N_THRESHOLD seam is si_config.dense_threshold
    here (0 keeps the default 2000; 1 sends every n past the dense level)."""
    import spectral_init_b200 as si
    lap, _ = _laplacian(ring(100))
    _, level = si.solve_eigenproblem_pub(lap, 2, 42, ctx=gpu_ctx)
    assert level == 0
    _, level = si.solve_eigenproblem_pub(lap, 2, 42, si.SpectralInitConfig(dense_threshold=1), ctx=gpu_ctx)
    assert level >= 1


@pytest.mark.parametrize("ds", ["blobs_50", "blobs_connected_2000"])
def test_b3_sign_convention(gpu_ctx, ds):
    import spectral_init_b200 as si
    from conftest import load_graph
    out = si.spectral_init(load_graph(ds), 2, 42, ctx=gpu_ctx)
    for c in range(2):
        col = out[:, c]
        assert col[int(np.argmax(np.abs(col)))] >= 0.0


def test_b4_multi_component_completeness(gpu_ctx):
    import spectral_init_b200 as si
    g = sp.block_diag([path(100), path(100)], format="csr").astype(np.float32)
    g.sort_indices()
    out = si.spectral_init(g, 2, 42, ctx=gpu_ctx).astype(np.float64)
    assert np.all(np.linalg.norm(out, axis=1) > 1e-9)


def test_b5_eigenvalues_non_negative(gpu_ctx):
    import spectral_init_b200 as si
    lap, sq = _laplacian(ring(500))
    r = si.lobpcg_solve(lap, 2, 42, False, sq, ctx=gpu_ctx)
    assert r is not None
    (vals, _), _ = r
    assert np.all(vals >= -1e-9)


def test_b6_lobpcg_converges_on_ring_2000(gpu_ctx):
    """Ring C_2000 (pairwise-degenerate spectrum).  The crate's test expects at
    least one warm restart of its linfa iteration; iterates are not pinned and
    this solver's block carries a guard vector, so the restart count is
    reported, not asserted: the pairs must pass the level gate, and at a tight
    tolerance the eigenvalues are the ring's 1 - cos(2 pi k / n)."""
    import spectral_init_b200 as si
    lap, sq = _laplacian(ring(2000))
    r = si.lobpcg_solve(lap, 2, 42, False, sq, ctx=gpu_ctx)
    assert r is not None
    (vals, vecs), restarts = r
    assert restarts >= 0
    assert O.max_eigenpair_residual(lap, vals, vecs) < 1e-5
    r = si.lobpcg_solve(lap, 2, 42, False, sq, si.SpectralInitConfig(tol=1e-10), ctx=gpu_ctx)
    assert r is not None
    (vals, _), _ = r
    exact = 1.0 - np.cos(2.0 * np.pi * np.array([0, 1, 1]) / 2000)
    assert np.all(np.abs(vals - exact) < 1e-9), (vals, exact)


def test_b7_rsvd_vectors_distinct(gpu_ctx):
    import spectral_init_b200 as si
    from conftest import load_csr
    _, vecs = si.rsvd_solve(load_csr("blobs_5000", "comp_b_laplacian.npz"), 2, 42, oversampling=61, ctx=gpu_ctx)
    v0, v1 = vecs[:, 0], vecs[:, 1]
    assert abs(v0 @ v1) / max(np.linalg.norm(v0) * np.linalg.norm(v1), 1e-300) < 0.99


def test_b8_sinv_nonzero(gpu_ctx):
    import spectral_init_b200 as si
    lap, _ = _laplacian(ring(2500))
    (vals, vecs), level = si.solve_eigenproblem_pub(lap, 2, 42, si.SpectralInitConfig(force_level=2), ctx=gpu_ctx)
    assert level == 2
    assert np.all(np.linalg.norm(vecs, axis=0) > 0.5)


# ---- failure paths, injected on the host -------------------------------------------------------
def test_iteration_cap_escalates_past_level1(gpu_ctx):
    """Level 1 capped at 3 iterations per pass cannot pass its gate on P_3000,
    so the chain moves on (src/solvers/mod.rs:70-224) and the level that
    answers passes its own gate; the answer matches the dense oracle."""
    import spectral_init_b200 as si
    lap = _path_lap(3000)
    cfg = si.SpectralInitConfig(max_iterations=3)
    (vals, vecs), level = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx)
    assert level >= 2
    gate = {2: 1e-6, 3: 1e-5, 4: 1e-2, 5: 1e-6}[level]
    assert O.max_eigenpair_residual(lap, vals, vecs) < gate
    ref = CERT.reference_eigenpairs(lap, 3, extra=6, dense_max=4000)
    assert np.all(np.abs(vals - ref.vals[:3]) < 1e-6)


def test_learned_start_fallback(gpu_ctx, monkeypatch):
    """The pass from the learned block capped at 2 iterations stalls; the
    solver restarts from the random block, converges, and reports that the
    accepted solve did not start from the learned block."""
    import spectral_init_b200 as si
    from spectral_init_b200.warm_start import WEIGHTS_PATH, WarmStartModel
    from conftest import load_csr
    if not WEIGHTS_PATH.exists():
        pytest.skip("no trained warm-start weights")
    lap = load_csr("blobs_connected_2000", "comp_b_laplacian.npz")
    model = WarmStartModel.load(ctx=gpu_ctx)
    model.attach()
    try:
        cfg = si.SpectralInitConfig(warm_start=si.WarmStart.LEARNED, dense_threshold=1)
        ((v_ok, _), lev_ok), _ = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx, return_report=True)
        monkeypatch.setenv("SPECTRAL_INIT_LEARNED_MAXITER", "2")
        ((vals, vecs), level), rep = si.solve_eigenproblem_pub(lap, 2, 42, cfg, ctx=gpu_ctx, return_report=True)
    finally:
        model.close()
    assert lev_ok == 1
    assert level == 1 and rep.learned_start == 0
    assert O.max_eigenpair_residual(lap, vals, vecs) < 1e-5
    assert np.all(np.abs(vals - v_ok) < 1e-6)


@pytest.mark.parametrize("n", [517, 1999])
def test_coop_tridiag_wait_timeout_recovers(gpu_ctx, monkeypatch, n):
    """Dense EVD with the single-launch tridiagonalisation's wait limit set to
    zero: its waits give up (an error word, no hang), every CTA leaves, and
    the multi-launch steps redo the matrix.  The result equals LAPACK's, and
    the recovery shows in the launch count."""
    import spectral_init_b200 as si
    from spectral_init_b200 import _lib
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    a = (a + a.T) / 2
    mat = sp.csr_matrix(a)
    w = np.linalg.eigvalsh(a)[:3]
    lib = _lib.load()
    l0 = lib.si_kernel_launches()
    v1, _ = si.dense_evd(mat, 3, ctx=gpu_ctx)
    plain = lib.si_kernel_launches() - l0
    monkeypatch.setenv("SPECTRAL_INIT_COOP_WAIT_NS", "0")
    l0 = lib.si_kernel_launches()
    v2, x2 = si.dense_evd(mat, 3, ctx=gpu_ctx)
    recovered = lib.si_kernel_launches() - l0
    scale = np.max(np.abs(w))
    assert np.max(np.abs(v1 - w)) <= 1e-9 * scale
    assert np.max(np.abs(v2 - w)) <= 1e-9 * scale
    assert np.max(np.abs(a @ x2 - x2 * v2)) <= 1e-8 * scale
    assert recovered > plain + n  # the steps path: several launches per column
