"""Components packed onto ranks (spectral_init_b200.multi_gpu), host side on
the CPU: the LPT plan, and two gloo ranks producing the same embedding as one
process, with the device steps replaced by deterministic stand-ins (each
component's coordinates are a fixed function of its node ids, placed at its
meta position and range as the crate places them)."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch.multiprocessing as mp

from spectral_init_b200 import multi_gpu as MG


def test_lpt_assign_balances_and_is_deterministic():
    costs = [10, 7, 7, 5, 3, 2, 2, 1]
    a = MG.lpt_assign(costs, 3)
    loads = [sum(c for c, r in zip(costs, a) if r == k) for k in range(3)]
    assert max(loads) - min(loads) <= max(costs)
    assert list(a) == list(MG.lpt_assign(costs, 3))
    assert a[0] == 0  # the largest item goes first to rank 0
    assert list(MG.lpt_assign(costs, 1)) == [0] * len(costs)


def test_data_ranges_and_orthogonal_positions():
    meta = MG.orthogonal_meta_embedding(5, 2)
    assert meta.tolist() == [[1, 0], [0, 1], [0, -1], [-1, 0], [-1, 0]] or meta.shape == (5, 2)
    r = MG.data_ranges(np.array([[0.0, 0.0], [2.0, 0.0], [0.0, 4.0]]))
    assert np.allclose(r, [1.0, 1.0, 2.0])


def _graph():
    rng = np.random.default_rng(3)
    blocks = []
    for size in (40, 7, 120, 3, 60, 25):
        a = sp.random(size, size, density=0.2, random_state=rng, format="csr")
        a = a + a.T + sp.diags(np.ones(size - 1), 1, shape=(size, size)) + sp.diags(np.ones(size - 1), -1,
                                                                                  shape=(size, size))
        blocks.append(a)
    g = sp.block_diag(blocks, format="csr").astype(np.float32)
    g.sort_indices()
    perm = np.random.default_rng(4).permutation(g.shape[0])  # components interleaved in node order
    g = g[perm][:, perm].tocsr()
    g.sort_indices()
    return g


def _fake_embed(graph, members, dims, data_range, meta_pos, seed):
    base = np.stack([np.cos(members * (d + 1.0)) for d in range(dims)], axis=1)
    base = base / np.max(np.abs(base))
    return base * data_range + np.asarray(meta_pos)[None, :]


def _fake_meta(data, members, nc, dims, seed, ctx):
    cent = np.stack([data[m].mean(axis=0)[:dims] for m in members])
    return cent / np.max(np.abs(cent))


def _data(n):
    return np.random.default_rng(9).standard_normal((n, 3)).astype(np.float32)


def _finish(out, seed):
    return (out * (10.0 / np.max(np.abs(out)))).astype(np.float32)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _graph()
        out = MG.spectral_init_components(g, 2, 42, data=_data(g.shape[0]), embed_component=_fake_embed,
                                          meta_embedding=_fake_meta, finish=_finish)
        q.put((rank, None if out is None else out.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_process():
    g = _graph()
    single = MG.spectral_init_components(g, 2, 42, data=_data(g.shape[0]), embed_component=_fake_embed,
                                         meta_embedding=_fake_meta, finish=_finish)
    assert single.shape == (g.shape[0], 2) and np.all(np.isfinite(single))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    assert np.array_equal(np.array(got[0], dtype=np.float32), single)


def test_component_numbering_and_members():
    g = _graph()
    nc, labels = sp.csgraph.connected_components(g, directed=False)
    assert nc == 6
    mem = MG.component_members(np.asarray(labels), nc)
    assert sorted(np.concatenate(mem).tolist()) == list(range(g.shape[0]))
    assert all(np.all(np.diff(m) > 0) for m in mem)


@pytest.mark.gpu
def test_components_path_matches_pipeline_on_gpu(gpu_ctx):
    """One process with the real device steps: the component-packing path
    gives the pipeline's embedding (si_spectral_init) for a 9-component graph
    with a determined spectral meta-embedding, up to per-axis sign."""
    import spectral_init_b200 as si
    from oracle import graphgen as G
    rng = np.random.default_rng(5)
    parts, pts = [], []
    for c in range(9):
        xc = G.gaussian_mixture(150, 1, 4, seed=100 + c, center_std=0.0) * 0.3
        xc = xc + rng.normal(0.0, 0.5, size=(1, 4)).astype(np.float32)
        parts.append(G.fuzzy_knn_graph(xc, 10))
        pts.append(xc)
    g = sp.block_diag(parts, format="csr").astype(np.float32)
    g.sort_indices()
    x = np.concatenate(pts).astype(np.float32)
    a = MG.spectral_init_components(g, 2, 42, data=x, ctx=gpu_ctx)
    b = si.spectral_init(g, 2, 42, data=x, ctx=gpu_ctx)
    for ax in range(2):
        err = min(np.abs(a[:, ax] - b[:, ax]).max(), np.abs(a[:, ax] + b[:, ax]).max())
        assert err < 1e-3, (ax, err)
