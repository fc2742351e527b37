"""Disconnected graphs across GPUs: components packed onto ranks.

The crate embeds the connected components of a disconnected graph one after
another (``embed_disconnected``, src/multi_component.rs:16-71, per component
``embed_single_component`` at :261-312).  The components are independent, so
with one process per GPU (``torch.distributed``, NCCL or gloo) they are packed
onto ranks by longest-processing-time-first on an estimated cost (stored
entries + nodes), each rank embeds its own components on its GPU through the C
ABI, and rank 0 gathers the coordinates once, places them and applies the
final scale and noise.  The meta-embedding (component positions and ranges)
is a small problem every rank computes identically.  No data-path collective
is needed besides the final gather; a single connected graph is not sharded
(``spectral_init`` on rank 0).

    from spectral_init_b200.multi_gpu import spectral_init_components
    emb = spectral_init_components(graph, 2, 42, data=points)   # rank 0: [n, 2]; other ranks: None
"""
from __future__ import annotations

import heapq

import numpy as np
import scipy.sparse as sp
from scipy.sparse import csgraph


def lpt_assign(costs, world: int) -> np.ndarray:
    """Rank of each item: items in decreasing cost (ties by index) go to the
    least-loaded rank (ties to the lowest rank).  Deterministic, so every rank
    computes the same plan."""
    costs = np.asarray(costs, dtype=np.float64)
    out = np.zeros(len(costs), dtype=np.int64)
    heap = [(0.0, r) for r in range(max(1, world))]
    heapq.heapify(heap)
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        load, r = heapq.heappop(heap)
        out[i] = r
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out


def component_members(labels: np.ndarray, nc: int):
    """Sorted node indices of each component (src/multi_component.rs:115-125)."""
    order = np.argsort(labels, kind="stable")
    bounds = np.searchsorted(labels[order], np.arange(nc + 1))
    return [order[bounds[c]:bounds[c + 1]] for c in range(nc)]


def orthogonal_meta_embedding(nc: int, dims: int) -> np.ndarray:
    """src/multi_component.rs:127-140: component c at +/- e_(c mod dims)."""
    m = np.zeros((nc, dims))
    for row in range(nc):
        m[row, row % dims] = 1.0 if row < dims else -1.0
    return m


def data_ranges(meta: np.ndarray) -> np.ndarray:
    """src/multi_component.rs:224-255: half the distance to the nearest other
    (distinct) component position; 1 when there is none."""
    nc = meta.shape[0]
    if nc == 1:
        return np.ones(1)
    d = np.sqrt(((meta[:, None, :] - meta[None, :, :]) ** 2).sum(axis=2))
    out = np.ones(nc)
    for c in range(nc):
        cand = d[c][(np.arange(nc) != c) & (d[c] > 0.0)]
        if cand.size:
            out[c] = cand.min() / 2.0
    return out


def _gpu_meta_embedding(data, members, nc, dims, seed, ctx):
    """src/multi_component.rs:143-220 on the device: centroids, Gaussian
    affinity, normalised Laplacian, its eigenvectors 1..dims scaled to max 1."""
    from . import api
    x = np.asarray(data, dtype=np.float32)
    cent = np.stack([x[m].astype(np.float64).sum(axis=0) * (1.0 / len(m)) if len(m) else np.zeros(x.shape[1])
                     for m in members])
    d2 = ((cent[:, None, :] - cent[None, :, :]) ** 2).sum(axis=2)
    aff = np.exp(-d2)
    np.fill_diagonal(aff, 0.0)
    deg = aff.sum(axis=1)
    inv = np.where(deg > 0, 1.0 / np.sqrt(np.where(deg > 0, deg, 1.0)), 0.0)
    lap = np.eye(nc) - inv[:, None] * aff * inv[None, :]
    (vals, vecs), _ = api.solve_eigenproblem_pub(sp.csr_matrix(lap), dims, seed, ctx=ctx)
    sel = api.select_eigenvectors(vals, vecs, dims)
    mx = float(np.max(np.abs(sel)))
    if mx == 0.0:
        raise api.InvalidGraph("invalid graph: spectral meta-embedding produced all-zero result")
    return sel / mx


def embed_component_gpu(graph, members, dims, data_range, meta_pos, seed, config, ctx):
    """``embed_single_component`` (src/multi_component.rs:261-312) through the
    C ABI: subgraph, device degrees and Laplacian, the eigensolver chain with
    the component's sqrt-degrees, selection, sign rule, scale to the range,
    translate to the position.  Tiny components collapse to the position."""
    import ctypes as C
    import torch
    from . import api
    from ._lib import SiReport
    from .warm_start import DeviceLaplacian
    size = len(members)
    if size < 2 * dims:
        return np.tile(np.asarray(meta_pos, dtype=np.float64), (size, 1))
    sub = graph[members][:, members].tocsr().astype(np.float32)
    sub.sort_indices()
    lap = DeviceLaplacian(sub, ctx=ctx, mode=int(config.compute_mode))
    k = dims + 1
    vals = (C.c_double * k)()
    vecs = torch.empty(size, k, dtype=torch.float64, device=f"cuda:{ctx.device}")
    level = C.c_int32(-1)
    rep = SiReport()
    cfg = config.to_c()
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_solve_eigenproblem(ctx.ptr, C.byref(lap.op()), dims, seed, lap.sqrt_deg.data_ptr(),
                                            C.byref(cfg), vals, vecs.data_ptr(), C.byref(level), C.byref(rep)))
    order = sorted(range(k), key=lambda i: vals[i])[1:dims + 1]
    coords = vecs[:, order].contiguous()
    ctx.check(ctx.lib.si_normalize_signs(ctx.ptr, coords.data_ptr(), size, dims))
    c = coords.cpu().numpy()
    mx = float(np.max(np.abs(c)))
    if mx > 0.0:
        c = c * (data_range / mx)
    return c + np.asarray(meta_pos, dtype=np.float64)[None, :]


def spectral_init_components(graph, n_components: int, seed: int, data=None, config=None, *, ctx=None,
                             embed_component=None, meta_embedding=None, finish=None):
    """``spectral_init`` (src/lib.rs:198-258) with the components of a
    disconnected graph spread over the ranks of the default process group
    (one process per GPU; a single process when no group is initialised).
    Returns the f32 ``[n, n_components]`` embedding on rank 0, None elsewhere.

    ``embed_component``, ``meta_embedding`` and ``finish`` replace the device
    steps (per-component embedding, spectral meta-embedding, final scale and
    noise); they exist so the host-side plan and gather can be tested without
    a GPU."""
    from . import api
    try:
        import torch.distributed as dist
        dist_on = dist.is_available() and dist.is_initialized()
    except Exception:
        dist, dist_on = None, False
    rank = dist.get_rank() if dist_on else 0
    world = dist.get_world_size() if dist_on else 1
    config = config or api.SpectralInitConfig()
    g = sp.csr_matrix(graph)
    n = g.shape[0]
    if embed_component is None:
        ctx = ctx or api.get_context()
        labels, nc = api.find_components(g, ctx=ctx)
    else:
        nc, labels = csgraph.connected_components(g, directed=False)
        # number components by their smallest node, as the crate's BFS does
        first = np.full(nc, n)
        np.minimum.at(first, labels, np.arange(n))
        remap = np.empty(nc, dtype=np.int64)
        remap[np.argsort(first, kind="stable")] = np.arange(nc)
        labels = remap[labels]
    labels = np.asarray(labels, dtype=np.int64)
    if n_components <= 0 or n == 0:
        raise api.InvalidGraph(f"spectral_init requires n > 0 and n_components > 0; got n={n}, "
                               f"n_components={n_components}")
    if n <= n_components:
        raise api.TooFewNodes(f"too few nodes: n={n} <= n_components={n_components}", n, n_components)
    if nc <= 1:
        if rank != 0:
            return None
        return api.spectral_init(g, n_components, seed, data=data, config=config, ctx=ctx)
    members = component_members(labels, nc)
    if nc > 2 * n_components:
        if data is None:
            raise api.InvalidGraph("invalid graph: data is required for spectral meta-embedding when "
                                   "n_conn_components > 2 * n_embedding_dims")
        meta = (meta_embedding or _gpu_meta_embedding)(data, members, nc, n_components, seed, ctx)
    else:
        meta = orthogonal_meta_embedding(nc, n_components)
    ranges = data_ranges(meta)
    row_nnz = np.diff(g.indptr)
    costs = [float(row_nnz[m].sum() + len(m)) for m in members]
    owner = lpt_assign(costs, world)
    embed = embed_component or (lambda gr, m, d, r, p, s: embed_component_gpu(gr, m, d, r, p, s, config, ctx))
    mine = {c: embed(g, members[c], n_components, ranges[c], meta[c], seed)
            for c in range(nc) if owner[c] == rank}
    if dist_on and world > 1:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(mine, gathered, dst=0)
        if rank != 0:
            return None
        parts = {}
        for d in gathered:
            parts.update(d)
    else:
        parts = mine
    out = np.zeros((n, n_components))
    for c in range(nc):
        out[members[c]] = parts[c]
    if finish is not None:
        return finish(out, seed)
    import torch
    dev = torch.device("cuda", ctx.device)
    x = torch.from_numpy(out).to(dev)
    y = torch.empty(n, n_components, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_scale_and_add_noise(ctx.ptr, x.data_ptr(), n, n_components, seed, y.data_ptr()))
    return y.cpu().numpy()
