"""Train the learned warm start on the GPU and write its weights.

    python -m spectral_init_b200.train_warm_start --graphs 2000 --epochs 6 \
        --out spectral_init_b200/warm_start_weights.bin

Training set: seeded Gaussian-mixture fuzzy-kNN graphs of the n=200k benchmark
family (n log-uniform in [10k, 200k], 5-100 clusters with anisotropic
covariances and Dirichlet(0.5) sizes, 10-100 dimensions, k in {10, 15, 30}),
built on the GPU.  Disconnected draws are skipped: the solve of a connected
graph is what the network starts.  Targets are the k+1 = 3 eigenvectors the
plain FP64 solver returns for n_components = 2.  Every step of the forward
pass, the subspace-projection loss, the backward pass and Adam runs in the
library's own kernels (``si_model_train_step``).  At the end the script
compares LOBPCG iterations from the random and the learned start on held-out
graphs and prints one JSON line per graph.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time

import numpy as np


def make_family_graph(rng, seed, device, n_min=10_000, n_max=200_000):
    import torch
    from . import synthetic
    n = int(math.exp(rng.uniform(math.log(n_min), math.log(n_max))))
    clusters = int(rng.integers(5, 101))
    dims = int(rng.integers(10, 101))
    k = int(rng.choice([10, 15, 30]))
    center_std = float(rng.uniform(1.0, 3.0))
    background = float(rng.uniform(0.0, 0.05))
    x = synthetic.gaussian_mixture_gpu(n, clusters, dims, seed, center_std, background, anisotropic=True,
                                       dirichlet_alpha=0.5, device=device)
    idx, dist = synthetic.knn_gpu(x, k)
    del x
    sigma, rho = synthetic.smooth_knn_gpu(dist, k)
    g = synthetic.fuzzy_graph_gpu(idx, dist, sigma, rho)
    torch.cuda.synchronize()
    return g, n, dict(n=n, clusters=clusters, dims=dims, k=k, center_std=center_std, background=background)


def n_components(ctx, g, n):
    import torch
    from ._lib import SiCsrF32
    labels = torch.empty(n, dtype=torch.int32, device=g[0].device)
    cnt = C.c_uint64(0)
    csr = SiCsrF32(n, int(g[1].numel()), g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr())
    ctx.check(ctx.lib.si_find_components(ctx.ptr, C.byref(csr), labels.data_ptr(), C.byref(cnt)))
    return int(cnt.value)


def solve(ctx, lap, precision, warm_start, seed=42, nc=2, learned_filter=0):
    """(vecs torch f64 [n, nc+1], report) from si_solve_eigenproblem."""
    import torch
    from ._lib import SiConfig, SiReport
    k = nc + 1
    cfg = SiConfig()
    ctx.lib.si_config_default(C.byref(cfg))
    cfg.precision = precision
    cfg.warm_start = warm_start
    cfg.learned_filter = learned_filter
    vals = (C.c_double * k)()
    vecs = torch.empty(lap.n, k, dtype=torch.float64, device=lap.v64.device)
    level = C.c_int32(-1)
    rep = SiReport()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.check(ctx.lib.si_solve_eigenproblem(ctx.ptr, C.byref(lap.op()), nc, seed, lap.sqrt_deg.data_ptr(),
                                            C.byref(cfg), vals, vecs.data_ptr(), C.byref(level), C.byref(rep)))
    return vecs, rep, level.value, time.perf_counter() - t0


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--graphs", type=int, default=2000)
    p.add_argument("--epochs", type=int, default=6)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--seed", type=int, default=1234)
    p.add_argument("--holdout", type=int, default=6)
    p.add_argument("--n-max", type=int, default=200_000)
    p.add_argument("--out", default=None)
    p.add_argument("--time-budget", type=float, default=1e9, help="stop generating after this many seconds")
    p.add_argument("--eval-1m", action="store_true",
                   help="also compare the starts on the held-out n=1M, k=15 benchmark graph")
    a = p.parse_args(argv)

    import torch
    from .api import SpectralError, get_context
    from .warm_start import WEIGHTS_PATH, DeviceLaplacian, WarmStartModel

    dev = torch.device("cuda", 0)
    ctx = get_context(0)
    rng = np.random.default_rng(a.seed)
    t_start = time.perf_counter()
    data = []
    skipped = 0
    for i in range(a.graphs):
        if time.perf_counter() - t_start > a.time_budget:
            break
        g, n, meta = make_family_graph(rng, a.seed * 100003 + i, dev, n_max=a.n_max)
        if n_components(ctx, g, n) != 1:
            skipped += 1
            continue
        lap = DeviceLaplacian((g[0], g[1], g[2], n), ctx=ctx)
        try:
            vecs, rep, level, _ = solve(ctx, lap, 0, 0)
        except SpectralError:
            skipped += 1
            continue
        if level != 1 or not rep.max_residual < 1e-5:
            skipped += 1
            continue
        lap.v64 = torch.zeros(1, dtype=torch.float64, device=dev)  # the network reads the f32 values only
        data.append((lap, vecs))
    t_gen = time.perf_counter() - t_start
    print(json.dumps({"phase": "data", "graphs": len(data), "skipped": skipped, "seconds": round(t_gen, 1)}),
          flush=True)

    model = WarmStartModel(a.seed, ctx=ctx)
    steps = 0
    t0 = time.perf_counter()
    for ep in range(a.epochs):
        order = rng.permutation(len(data))
        losses = []
        lr = a.lr * (0.5 * (1 + math.cos(math.pi * ep / max(1, a.epochs))))
        for j in order:
            lap, vecs = data[j]
            losses.append(model.train_step(lap, vecs, seed=int(rng.integers(1 << 31)), lr=lr))
            steps += 1
        print(json.dumps({"phase": "train", "epoch": ep, "lr": lr, "loss_mean": float(np.mean(losses)),
                          "loss_median": float(np.median(losses))}), flush=True)
    t_train = time.perf_counter() - t0
    out = a.out or str(WEIGHTS_PATH)
    model.save(out)
    print(json.dumps({"phase": "saved", "path": out, "steps": steps, "seconds": round(t_train, 1)}), flush=True)
    del data

    # held-out comparison: random vs learned start, mixed precision
    model.attach()
    for h in range(a.holdout):
        g, n, meta = make_family_graph(rng, 777_000 + h, dev, n_max=a.n_max)
        if n_components(ctx, g, n) != 1:
            continue
        lap = DeviceLaplacian((g[0], g[1], g[2], n), ctx=ctx)
        row = dict(meta)
        try:
            for name, ws, lf in (("random", 0, 0), ("learned", 1, 0), ("learned_filtered", 1, 1)):
                solve(ctx, lap, 1, ws, learned_filter=lf)
                _, rep, level, sec = solve(ctx, lap, 1, ws, learned_filter=lf)
                row[name] = {"iterations": rep.iterations, "s": round(sec, 4), "level": level,
                             "residual": rep.max_residual}
        except SpectralError as e:
            row["error"] = str(e)
        print(json.dumps({"phase": "holdout", **row}), flush=True)
    if a.eval_1m:
        from . import synthetic
        n = 1_000_000
        x = synthetic.gaussian_mixture_gpu(n, 100, 50, 42, 2.0, 0.05, device=dev)
        idx, dist = synthetic.knn_gpu(x, 15)
        del x
        sigma, rho = synthetic.smooth_knn_gpu(dist, 15)
        g = synthetic.fuzzy_graph_gpu(idx, dist, sigma, rho)
        del idx, dist
        lap = DeviceLaplacian((g[0], g[1], g[2], n), ctx=ctx)
        row = {"n": n, "clusters": 100, "dims": 50, "k": 15, "center_std": 2.0, "background": 0.05}
        for name, ws, lf in (("random", 0, 0), ("learned", 1, 0), ("learned_filtered", 1, 1)):
            solve(ctx, lap, 1, ws, learned_filter=lf)
            _, rep, level, sec = solve(ctx, lap, 1, ws, learned_filter=lf)
            row[name] = {"iterations": rep.iterations, "s": round(sec, 4), "level": level,
                         "residual": rep.max_residual, "learned_used": rep.learned_start}
        print(json.dumps({"phase": "heldout_1m", **row}), flush=True)
    model.close()


if __name__ == "__main__":
    main()
