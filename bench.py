#!/usr/bin/env python3
"""Benchmark of the spectral-init eigensolve path on B200.

Workload: synthetic UMAP fuzzy-kNN graph, n = 1,000,000 points of a
100-cluster Gaussian mixture in 50-D plus 5% uniform background, k = 15,
n_components = 2 (the crate's default embedding), seed 42.

One step = one eigensolve (solve_eigenproblem: Chebyshev-filtered start,
block LOBPCG, Rayleigh-Ritz refinement, FP64 residual gate <= 1e-5) with the
Laplacian already resident in HBM; step i solves with seed --seed + i, the
same seeds in every leg (the iteration count moves by tens of percent with
the random start).  `value` is the mean device time of the learned-start
mixed-precision solve (f32 bulk + f64 refinement) at --tol (1e-7, where the
subspace meets 1e-4 against the certified oracle); the plain FP64 solve at the
crate's 1e-5 and at --tol, the random-start mixed solve, the SpMM bandwidth
(the roofline kernel), the end-to-end C-ABI call with host buffers, and the
CPU baseline (the restated reference path on the host cores) are reported
beside it.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
    python bench.py --spmm-profile      # small SpMM-only run for ncu captures
    python bench.py --profile-solve [--solve-seed S --profile-repeat R --block-size B --switch-tol T]
    python bench.py --configs | --components | --dense | --learned-eval G | --accuracy-sweep
    python bench.py --cpu-only --cpu-threads T   # the CPU baseline alone
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "eigensolve s at n=1M (resid≤1e-5): learned+FP32 vs plain FP64 GPU; SpMM GB/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=1_000_000)
    p.add_argument("--k", type=int, default=15)
    p.add_argument("--nc", type=int, default=2)
    p.add_argument("--clusters", type=int, default=100)
    p.add_argument("--dims", type=int, default=50)
    p.add_argument("--center-std", type=float, default=2.0)
    p.add_argument("--background", type=float, default=0.05)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--spmm-reps", type=int, default=40)
    p.add_argument("--tol", type=float, default=1e-7,
                   help="LOBPCG tolerance of the mixed / learned legs (the headline): tight enough that their "
                        "subspace is within 1e-4 of the FP64 oracle on this graph; the plain FP64 leg runs at "
                        "the crate's 1e-5 (the drop-in)")
    p.add_argument("--switch-tol", type=float, default=0.0,
                   help="mixed precision: residual at which the f32 phase hands over to f64 (0: the library default)")
    p.add_argument("--learned-filter", type=int, default=1,
                   help="1 (default): apply the Chebyshev start filter to the learned block as well (measured at "
                        "the headline tolerance: 204 instead of 328 iterations); 0: the predicted block as is")
    p.add_argument("--no-oracle", action="store_true", help="skip the CPU ARPACK accuracy oracle")
    p.add_argument("--accuracy-sweep", action="store_true",
                   help="one JSON line: mixed/learned/FP64 solves at several tolerances, time and error vs the oracle")
    p.add_argument("--cpu-threads", type=int, default=0, help="threads of the CPU baseline (0: all)")
    p.add_argument("--cpu-only", action="store_true",
                   help="only the CPU baseline (one converged solve per step), for the 1-thread measurement")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-learned", action="store_true", help="skip the learned warm-start leg")
    p.add_argument("--solve-seed", type=int, default=None, help="eigensolver seed (default: --seed)")
    p.add_argument("--profile-repeat", type=int, default=1,
                   help="with --profile-solve: also time each leg this many times (same seed)")
    p.add_argument("--block-size", type=int, default=0,
                   help="LOBPCG block width (wanted pairs plus guard vectors; 0: the solver's choice)")
    p.add_argument("--spmm-profile", action="store_true", help="SpMM launches only (n=--n), for ncu")
    p.add_argument("--spmm-prec", choices=["both", "f64", "f32"], default="both",
                   help="with --spmm-profile: which SpMM precision to run")
    p.add_argument("--components", action="store_true",
                   help="the batched multi-component workload instead: 500 disconnected fuzzy-kNN components "
                        "(sizes log-uniform in [20, 100k], 1-10 clusters in 20-D), full pipeline, one JSON line")
    p.add_argument("--n-comp", type=int, default=500)
    p.add_argument("--configs", action="store_true",
                   help="the parity configurations instead: the n=200k family graph (FP64 / mixed / learned) and "
                        "the n=1M graph with n_components=8 and the rSVD path; one JSON line each")
    p.add_argument("--dense", action="store_true",
                   help="the device dense eigensolver (level 0) at n = 300 / 1000 / 1900 instead, one JSON line")
    p.add_argument("--learned-eval", type=int, default=0, metavar="G",
                   help="one JSON line: learned vs random start (mixed precision, --tol) on G held-out graphs of the "
                        "benchmark family (seeds --seed+1 .. --seed+G), iterations and device time")
    p.add_argument("--profile-solve", action="store_true",
                   help="one FP64 and one mixed eigensolve only (after one warm-up each), for ncu launch lists")
    return p.parse_args()


def workload_name(a) -> str:
    return (f"fuzzy-kNN graph n={a.n} k={a.k}: {a.clusters}-cluster Gaussian mixture in {a.dims}-D "
            f"(centers N(0,{a.center_std}^2 I), unit variance) + {a.background:.0%} uniform background, "
            f"seed {a.seed}; n_components={a.nc}")


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile(prefix="si_clocks_", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.close()
        rows = [r.split(",") for r in Path(self.tmp.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def graph_cache_path(a) -> Path:
    tag = f"n{a.n}_k{a.k}_c{a.clusters}_d{a.dims}_s{a.center_std}_b{a.background}_seed{a.seed}"
    return Path(tempfile.gettempdir()) / f"si_bench_graph_{tag}.npz"


def make_graph(a, device, rank=0):
    """(indptr i64, indices i32, data f32) torch CUDA tensors of the workload graph."""
    import numpy as np
    import torch
    from spectral_init_b200 import synthetic
    path = graph_cache_path(a)
    if rank == 0 and path.exists():
        z = np.load(path)
        return (torch.from_numpy(z["indptr"]).to(device), torch.from_numpy(z["indices"]).to(device),
                torch.from_numpy(z["data"]).to(device))
    seed = a.seed + rank
    x = synthetic.gaussian_mixture_gpu(a.n, a.clusters, a.dims, seed, a.center_std, a.background, device=device)
    idx, dist = synthetic.knn_gpu(x, a.k)
    del x
    sigma, rho = synthetic.smooth_knn_gpu(dist, a.k)
    g = synthetic.fuzzy_graph_gpu(idx, dist, sigma, rho)
    del idx, dist
    torch.cuda.synchronize()
    if rank == 0:
        try:
            np.savez(path, indptr=g[0].cpu().numpy(), indices=g[1].cpu().numpy(), data=g[2].cpu().numpy())
        except OSError:
            pass
    return g


# ---------------------------------------------------------------------------------------------
def dist_helpers(dist, device):
    """(barrier, max_over_ranks) for one process per GPU; with dist None (one
    process) both are no-ops.  Times are reduced on the device of the
    backend (NCCL: the rank's GPU; gloo: the CPU)."""
    import torch

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def run_ours(a):
    import numpy as np
    import torch

    import spectral_init_b200 as si
    from spectral_init_b200 import _lib
    from spectral_init_b200._lib import SiConfig, SiCsrF32, SiOperator, SiReport

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    barrier, max_over_ranks = dist_helpers(dist, dev)
    try:
        _run_ours_body(a, rank, world, local, dev, barrier, max_over_ranks)
    finally:
        if dist is not None:
            dist.destroy_process_group()


def _run_ours_body(a, rank, world, local, dev, barrier, max_over_ranks):
    import numpy as np
    import torch

    import spectral_init_b200 as si
    from spectral_init_b200 import _lib
    from spectral_init_b200._lib import SiConfig, SiCsrF32, SiOperator, SiReport

    ctx = si.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.si_ctx_stream(ctx.ptr), device=dev)

    t0 = time.time()
    indptr, indices, data = make_graph(a, dev, rank)
    n = a.n
    nnz = int(indices.numel())
    t_gen = time.time() - t0
    g = SiCsrF32(n, nnz, indptr.data_ptr(), indices.data_ptr(), data.data_ptr())
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    ncomp = C.c_uint64(0)
    torch.cuda.synchronize()
    ctx.check(lib.si_find_components(ctx.ptr, C.byref(g), labels.data_ptr(), C.byref(ncomp)))
    deg = torch.empty(n, dtype=torch.float64, device=dev)
    sq = torch.empty_like(deg)
    ctx.check(lib.si_compute_degrees(ctx.ptr, C.byref(g), 0, deg.data_ptr(), sq.data_ptr()))
    inv = torch.where(sq > 0, 1.0 / sq, torch.zeros_like(sq))
    v64 = torch.empty(nnz, dtype=torch.float64, device=dev)
    v32 = torch.empty(nnz, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    ctx.check(lib.si_build_laplacian(ctx.ptr, C.byref(g), inv.data_ptr(), v64.data_ptr(), v32.data_ptr()))
    op = SiOperator(n, nnz, indptr.data_ptr(), indices.data_ptr(), v64.data_ptr(), v32.data_ptr(), 1.0)

    # ---- SpMM (the roofline kernel): the prepared operator, kernels back to back on the stream ----
    plan = C.c_void_p()
    ctx.check(lib.si_operator_plan_create(ctx.ptr, C.byref(op), C.byref(plan)))

    def time_spmm(x, y, f32: bool, reps: int):
        fn = lib.si_spmm_planned_f32 if f32 else lib.si_spmm_planned
        for _ in range(3):
            ctx.check(fn(ctx.ptr, plan, x.data_ptr(), y.data_ptr(), 4))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            ctx.check(fn(ctx.ptr, plan, x.data_ptr(), y.data_ptr(), 4))
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    gen = torch.Generator(device=dev)
    gen.manual_seed(1)
    x64 = torch.randn(n, 4, dtype=torch.float64, device=dev, generator=gen)
    y64 = torch.empty_like(x64)
    x32 = x64.float()
    y32 = torch.empty_like(x32)
    torch.cuda.synchronize()
    run64 = not (a.spmm_profile and a.spmm_prec == "f32")
    run32 = not (a.spmm_profile and a.spmm_prec == "f64")
    ms64 = time_spmm(x64, y64, False, a.spmm_reps) if run64 else float("nan")
    ms32 = time_spmm(x32, y32, True, a.spmm_reps) if run32 else float("nan")
    bytes64 = nnz * (4 + 8) + (n + 1) * 8 + 2 * n * 4 * 8
    bytes32 = nnz * (4 + 4) + (n + 1) * 8 + 2 * n * 4 * 4
    gbs64 = bytes64 / (ms64 * 1e-3) / 1e9
    gbs32 = bytes32 / (ms32 * 1e-3) / 1e9
    lib.si_operator_plan_destroy(plan)
    if a.spmm_profile:
        print(json.dumps({"spmm_profile": True, "n": n, "nnz": nnz, "ms_f64": ms64, "ms_f32": ms32,
                          "gbs_f64": gbs64, "gbs_f32": gbs32}))
        return

    # ---- eigensolves ------------------------------------------------------------------------
    k = a.nc + 1

    # learned warm start: the committed network weights, when present
    model = None
    if not a.no_learned:
        from spectral_init_b200.warm_start import WEIGHTS_PATH, WarmStartModel
        if WEIGHTS_PATH.exists():
            model = WarmStartModel.load(ctx=ctx)
            model.attach()
    # (name, precision, warm start, tol): the plain FP64 solve at the crate's
    # tolerance is the drop-in; the mixed / learned legs run at --tol
    legs = [("fp64", 0, 0, 0.0), ("mixed", 1, 0, a.tol)]
    if model is not None:
        legs.append(("learned", 1, 1, a.tol))
    if a.tol < 1e-5:
        legs.append(("fp64_same_tol", 0, 0, a.tol))
    head = "learned" if model is not None else "mixed"

    base_seed = a.seed if a.solve_seed is None else a.solve_seed

    def solve(precision: int, warm: int = 0, tol: float = 0.0, switch_tol: float | None = None,
              learned_filter: int | None = None, seed: int | None = None):
        cfg = SiConfig()
        lib.si_config_default(C.byref(cfg))
        cfg.precision = precision
        cfg.warm_start = warm
        cfg.tol = tol
        cfg.mixed_switch_tol = a.switch_tol if switch_tol is None else switch_tol
        cfg.learned_filter = a.learned_filter if learned_filter is None else learned_filter
        cfg.block_size = a.block_size
        vals = (C.c_double * k)()
        vecs = torch.empty(n, k, dtype=torch.float64, device=dev)
        level = C.c_int32(-1)
        rep = SiReport()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = lib.si_solve_eigenproblem(ctx.ptr, C.byref(op), a.nc, base_seed if seed is None else seed,
                                       sq.data_ptr(), C.byref(cfg), vals,
                                       vecs.data_ptr(), C.byref(level), C.byref(rep))
        e1.record(stream)
        e1.synchronize()
        ctx.check(st)
        return e0.elapsed_time(e1), list(vals), vecs, level.value, rep

    if a.profile_solve:
        out = {}
        for name, prec, warm, tol in legs:
            solve(prec, warm, tol)
            if a.profile_repeat > 1:
                reps = [solve(prec, warm, tol) for _ in range(a.profile_repeat)]
                out[name + "_repeat_ms"] = [round(r[0], 2) for r in reps]
            ms, vals, _, level, rep = solve(prec, warm, tol)
            out[name] = {"ms": ms, "iterations": rep.iterations, "fp32_iterations": rep.fp32_iterations,
                         "restarts": rep.restarts, "spmm_calls": rep.spmm_calls, "level": level,
                         "max_residual": rep.max_residual, "learned_start": rep.learned_start}
        print(json.dumps({"profile_solve": True, "n": n, "nnz": nnz, **out}))
        return

    oracle = None
    if rank == 0 and world == 1 and not a.no_oracle:
        oracle = host_oracle(a, indptr, indices, data, k)

    if a.accuracy_sweep:
        rows = []
        for name, prec, warm in (("mixed", 1, 0), ("learned", 1, 1), ("fp64", 0, 0)):
            if warm and model is None:
                continue
            for tol in (1e-5, 3e-6, 1e-6, 3e-7, 1e-7, 3e-8, 1e-8):
                solve(prec, warm, tol)
                ms, vals, vecs, level, rep = solve(prec, warm, tol)
                r = {"leg": name, "tol": tol, "ms": ms, "iterations": rep.iterations,
                     "fp32_iterations": rep.fp32_iterations, "max_residual": rep.max_residual,
                     "learned_start": rep.learned_start}
                if oracle is not None:
                    r["vs_oracle"] = oracle_errors(oracle, vals, vecs)
                rows.append(r)
                print(json.dumps(r), flush=True)
        # at the headline tolerance: where the f32 phase hands over, and the start filter on the learned block
        for name, prec, warm in (("mixed", 1, 0), ("learned", 1, 1)):
            if warm and model is None:
                continue
            for sw in (1e-4, 1e-5, 3e-6):
                for lf in ((0, 1) if warm else (0,)):
                    solve(prec, warm, a.tol, sw, lf)
                    ms, vals, vecs, level, rep = solve(prec, warm, a.tol, sw, lf)
                    r = {"leg": name, "tol": a.tol, "switch_tol": sw, "learned_filter": lf, "ms": ms,
                         "iterations": rep.iterations, "fp32_iterations": rep.fp32_iterations,
                         "max_residual": rep.max_residual, "learned_start": rep.learned_start}
                    if oracle is not None:
                        r["vs_oracle"] = oracle_errors(oracle, vals, vecs)
                    rows.append(r)
                    print(json.dumps(r), flush=True)
        print(json.dumps({"accuracy_sweep": True, "n": n, "nnz": nnz, "rows": rows,
                          "oracle": None if oracle is None else oracle["summary"]}))
        return

    # every leg solves the same seeds, one per timed step: LOBPCG's iteration
    # count varies by tens of percent with the random start, so a single seed
    # would rank the legs by luck
    step_seeds = [base_seed + i for i in range(a.steps)]
    results = {}
    clocks = None
    launches_per_step = None
    for name, prec, warm, tol in legs:
        for w in range(a.warmup):
            solve(prec, warm, tol, seed=base_seed + 1000 + w)
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if name == head else None
        if sampler:
            sampler.start()
        l0 = lib.si_kernel_launches()
        times, iters, restarts, spmms, last = [], [], [], [], None
        for sd in step_seeds:
            ms, vals, vecs, level, rep = solve(prec, warm, tol, seed=sd)
            times.append(ms)
            iters.append(rep.iterations)
            restarts.append(rep.restarts)
            spmms.append(rep.spmm_calls)
            last = (vals, vecs, level, rep)
        torch.cuda.synchronize()
        barrier()
        if sampler:
            clocks = sampler.stop()
            launches_per_step = (lib.si_kernel_launches() - l0) / a.steps
        ms_mean = max_over_ranks(statistics.mean(times))
        vals, vecs, level, rep = last
        results[name] = {"ms": ms_mean, "ms_all": times, "iterations_all": iters, "restarts_all": restarts,
                         "spmm_calls_all": spmms,
                         "iterations_mean": statistics.mean(iters), "tol": tol if tol > 0 else 1e-5,
                         "eigenvalues": vals,
                         "level": level, "iterations": rep.iterations, "fp32_iterations": rep.fp32_iterations,
                         "restarts": rep.restarts, "max_residual": rep.max_residual,
                         "learned_start": rep.learned_start, "vecs": vecs}
        if oracle is not None:
            results[name]["vs_oracle"] = oracle_errors(oracle, vals, vecs)

    # agreement of the headline solve with the plain FP64 solve: largest principal-angle sine, eigenvalues
    qa, _ = torch.linalg.qr(results["fp64"]["vecs"])
    qb, _ = torch.linalg.qr(results[head]["vecs"])
    sin_theta = float(torch.linalg.matrix_norm(qb - qa @ (qa.T @ qb), ord=2))
    ev64 = np.array(results["fp64"]["eigenvalues"])
    evm = np.array(results[head]["eigenvalues"])
    ev_rel = float(np.max(np.abs(evm - ev64) / np.maximum(np.abs(ev64), 1e-300)))

    # ---- end to end through the C ABI with host buffers ----------------------------------------
    e2e = None
    if not a.no_e2e:
        h_ip = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
        h_ix = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
        h_dv = torch.empty(nnz, dtype=torch.float32, pin_memory=True)
        h_out = torch.empty(n, a.nc, dtype=torch.float32, pin_memory=True)
        h_ip.copy_(indptr)
        h_ix.copy_(indices)
        h_dv.copy_(data)
        hg = SiCsrF32(n, nnz, h_ip.data_ptr(), h_ix.data_ptr(), h_dv.data_ptr())
        cfg = SiConfig()
        lib.si_config_default(C.byref(cfg))
        cfg.precision = 1
        cfg.warm_start = 1 if head == "learned" else 0
        cfg.tol = a.tol
        rep = SiReport()

        def call(sd):
            t = time.perf_counter()
            ctx.check(lib.si_spectral_init(ctx.ptr, C.byref(hg), a.nc, sd, None, 0, C.byref(cfg),
                                           h_out.data_ptr(), C.byref(rep)))
            return time.perf_counter() - t

        for w in range(max(1, min(a.warmup, 2))):
            call(base_seed + 1000 + w)
        barrier()
        ts = [call(sd) for sd in step_seeds]
        barrier()
        e2e = {"value": max_over_ranks(statistics.mean(ts)), "unit": "s",
               "h2d_bytes_per_step": (n + 1) * 8 + nnz * 8, "d2h_bytes_per_step": n * a.nc * 4,
               "what": "si_spectral_init (C ABI): host CSR upload, validation, components, degrees, Laplacian, "
                       "mixed-precision eigensolve, selection, signs, scaling + noise, result download; "
                       "wall clock around the synchronous call"}

    # ---- CPU baseline (rank 0, N=1) ---------------------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_sample(a, indptr, indices, data)

    peaks, peak_src = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    traffic = None
    tfile = ROOT / "profiles" / "spmm_traffic.json"
    if tfile.exists():
        t = json.loads(tfile.read_text())
        # measured DRAM bytes per f32 launch, scaled to this graph by bytes of the same formula
        if "dram_bytes_per_algorithmic_byte_f32" in t:
            traffic = t["dram_bytes_per_algorithmic_byte_f32"] * bytes32
    if rank != 0:
        return
    value_s = results[head]["ms"] / 1e3

    def leg(name):
        return {k2: v for k2, v in results[name].items() if k2 != "vecs"}

    line = {
        "metric": METRIC,
        "value": value_s,
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": results[head]["ms"],
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 SpMM/LOBPCG bulk + f64 Gram/Rayleigh-Ritz/refinement",
        "data": "synthetic (seeded Gaussian-mixture fuzzy-kNN graph built on the GPU)",
        "config": {"workload": workload_name(a), "n": n, "nnz": nnz, "connected_components": int(ncomp.value),
                   "block_columns": 4, "l2": "inputs larger than L2 (Laplacian "
                   f"{(nnz * 12 + (n + 1) * 8) / 1e6:.0f} MB f64 / {(nnz * 8 + (n + 1) * 8) / 1e6:.0f} MB f32)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "graph_build_s": round(t_gen, 2),
                   "tol_value_leg": a.tol, "tol_fp64_leg": 1e-5, "solve_seeds": step_seeds,
                   "warm_start": ("learned (committed network weights, trained on the n=10k-200k family)"
                                  + (", Chebyshev-filtered" if a.learned_filter else "")
                                  if head == "learned" else "random (no network weights found)")},
        **{name: leg(name) for name in results},
        "speedup_mixed_vs_fp64": results["fp64"]["ms"] / results["mixed"]["ms"],
        "speedup_value_vs_fp64": results["fp64"]["ms"] / results[head]["ms"],
        **({"speedup_value_vs_fp64_same_tol": results["fp64_same_tol"]["ms"] / results[head]["ms"]}
           if "fp64_same_tol" in results else {}),
        "value_vs_fp64": {"leg": head, "sin_theta_max": sin_theta, "eigenvalue_rel_diff_max": ev_rel},
        "value_vs_oracle": (None if oracle is None else
                            {"leg": head, **results[head]["vs_oracle"], "oracle": oracle["summary"]}),
        "spmm": {"ms_f64": ms64, "ms_f32": ms32, "gbs_f64": gbs64, "gbs_f32": gbs32,
                 "algorithmic_bytes_f64": bytes64, "algorithmic_bytes_f32": bytes32,
                 "bytes_formula": "nnz*(4 idx + s_val) + (n+1)*8 indptr + 2*n*4*s_x (x read, y written; 4 columns)"},
        "roofline": {"bound": "hbm", "kernel": "f32 SpMM, 4 columns (the autotuned kernel; ncu summary in profiles/)",
                     "achieved": gbs32, "peak": hbm, "unit": "GB/s", "frac": gbs32 / hbm,
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                     else "fallback 6.65 TB/s", "traffic": traffic},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches_per_step,
        "clocks": clocks,
    }
    print(json.dumps(line))


def host_oracle(a, indptr, indices, data, k):
    """The FP64 accuracy oracle on the host: the crate's Laplacian built on the
    CPU from the graph, ARPACK to machine precision (k + 6 pairs), residuals
    and the Davis-Kahan certificate."""
    import numpy as np
    from oracle import certified as CERT
    from oracle import cpu_baseline as CB
    t0 = time.time()
    op, _ = CB.laplacian_operator(indptr.cpu().numpy(), indices.cpu().numpy(), data.cpu().numpy(), a.n)
    ref = CERT.reference_eigenpairs_operator(op.apply, a.n, k, extra=6)
    secs = time.time() - t0
    gap = CERT.gap_after(ref, k)
    summary = {"method": ref.method, "seconds": round(secs, 1), "eigenvalues": [float(v) for v in ref.vals],
               "max_residual": float(np.max(ref.residuals)), "gap_k": gap,
               "sin_theta_bound": float(np.max(ref.residuals[:k]) / gap)}
    return {"ref": ref, "summary": summary}


def oracle_errors(oracle, vals, vecs):
    from oracle import certified as CERT
    c = CERT.compare(vals, vecs.cpu().numpy(), oracle["ref"])
    return {"sin_theta": c["sin_theta_max"], "sin_theta_subspace": c["sin_theta_subspace"],
            "eig_rel_max": c["eig_rel_max"], "eig_abs0": c["eig_abs0"]}


def cpu_baseline_sample(a, indptr, indices, data):
    """The restated CPU path on this host (OpenMP C SpMM + numpy LOBPCG), one
    solve run to completion and timed (the crate's Laplacian is built on the CPU
    first, outside the timed solve)."""
    from oracle import cpu_baseline as CB
    if a.cpu_threads > 0:
        CB.set_threads(a.cpu_threads)
    op, sqh = CB.laplacian_operator(indptr.cpu().numpy(), indices.cpu().numpy(), data.cpu().numpy(), a.n)
    spmm_s = CB.time_spmm(op, a.nc + 1, reps=3)
    res = CB.solve_measured(op, a.nc, a.seed, sqh)
    nnz = len(op.indices)
    bytes_k3 = nnz * 12 + (a.n + 1) * 8 + 2 * a.n * (a.nc + 1) * 8
    return {"value": res["seconds"], "unit": "s", "cores": CB.threads(), "kind": "port",
            "host": host_cpu(),
            "sample": (f"one complete crate Level-1 solve restated on the CPU (f64, block of {a.nc + 1}: random start, "
                       f"Chebyshev filter, LOBPCG with warm restarts, Rayleigh-Ritz, residual gate), measured to "
                       f"{'convergence' if res['converged'] else 'its end (not converged)'}: "
                       f"{res['iterations']} iterations, max residual {res['max_residual']:.2e}"),
            "iterations": res["iterations"], "restarts": res["restarts"], "converged": res["converged"],
            "spmm_s_k3": spmm_s, "spmm_gbs_k3": bytes_k3 / spmm_s / 1e9}


def host_cpu():
    try:
        model = next((ln.split(":", 1)[1].strip() for ln in Path("/proc/cpuinfo").read_text().splitlines()
                      if ln.startswith("model name")), "unknown")
    except OSError:
        model = "unknown"
    return {"nproc": os.cpu_count(), "model": model}


def run_reference(a):
    """The reference arm: the restated CPU path on this host for the same
    workload, metric and unit (rank 0 only).  Each timed step is one complete
    Level-1 solve (random start, Chebyshev filter, LOBPCG with warm restarts,
    Rayleigh-Ritz, residual gate) on the crate's Laplacian built on the CPU;
    the warm-up steps run the same code for one second each."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    from oracle import cpu_baseline as CB
    if a.cpu_threads > 0:
        CB.set_threads(a.cpu_threads)
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    indptr, indices, data = make_graph(a, dev, 0)
    n = a.n
    op, sqh = CB.laplacian_operator(indptr.cpu().numpy(), indices.cpu().numpy(), data.cpu().numpy(), n)
    base_seed = a.seed if a.solve_seed is None else a.solve_seed
    for w in range(a.warmup):
        CB.solve_timed(op, a.nc, base_seed + 1000 + w, sqh, budget_s=1.0)
    # one solve seed per step, the seeds the GPU arm uses; a complete CPU solve
    # takes about a minute at n = 1M, so at most three are timed (the line's
    # `steps` says how many)
    n_timed = max(1, min(a.steps, 3))
    samples = [CB.solve_measured(op, a.nc, base_seed + i, sqh) for i in range(n_timed)]
    val = statistics.mean(s["seconds"] for s in samples)
    s0 = samples[-1]
    conv = all(x["converged"] for x in samples)
    cpu = {"value": val, "unit": "s", "cores": CB.threads(), "kind": "port", "host": host_cpu(),
           "sample": (f"per step one complete crate Level-1 solve restated on the CPU (f64, block of {a.nc + 1}), "
                      f"measured to {'convergence' if conv else 'its end'}: "
                      f"{s0['iterations']} iterations, max residual {s0['max_residual']:.2e}"),
           "iterations": s0["iterations"], "restarts": s0["restarts"], "converged": conv,
           "seconds_all": [x["seconds"] for x in samples], "iterations_all": [x["iterations"] for x in samples],
           "solve_seeds": [base_seed + i for i in range(n_timed)]}
    line = {"metric": METRIC, "value": val, "unit": "s", "higher_is_better": False, "impl": "reference",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": n_timed, "warmup": a.warmup,
            "ms_per_step": val * 1e3, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian-mixture fuzzy-kNN graph)",
            "config": {"workload": workload_name(a), "n": n, "nnz": int(len(op.indices))},
            "cpu_baseline": cpu,
            "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_cpu_only(a):
    """One JSON line: the CPU baseline alone (--steps complete solves at
    --cpu-threads threads), for the single-thread measurement."""
    import torch
    indptr, indices, data = make_graph(a, torch.device("cuda", 0), 0)
    rows = [cpu_baseline_sample(a, indptr, indices, data) for _ in range(max(1, a.steps))]
    print(json.dumps({"cpu_only": True, "workload": workload_name(a), "threads": rows[0]["cores"],
                      "value": statistics.mean(r["value"] for r in rows), "unit": "s", "samples": rows}))


def run_components(a):
    """The multi-component workload: si_spectral_init_device on the block-diagonal
    graph with its points (spectral meta-embedding), device-timed, per-component
    residual gate reported through the worst component."""
    import numpy as np
    import torch
    import spectral_init_b200 as si
    from spectral_init_b200 import synthetic
    from spectral_init_b200._lib import SiConfig, SiCsrF32, SiReport
    dev = torch.device("cuda", 0)
    ctx = si.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.si_ctx_stream(ctx.ptr), device=dev)
    t0 = time.time()
    ip, ix, dv, n, pts, sizes = synthetic.multi_component_graph_gpu(a.n_comp, 20, 100_000, 20, 15, a.seed,
                                                                     device=dev)
    t_gen = time.time() - t0
    nnz = int(ix.numel())
    g = SiCsrF32(n, nnz, ip.data_ptr(), ix.data_ptr(), dv.data_ptr())
    out = torch.empty(n, a.nc, dtype=torch.float32, device=dev)
    results = {}
    clocks = None
    for prec, name in ((0, "fp64"), (1, "mixed")):
        cfg = SiConfig()
        lib.si_config_default(C.byref(cfg))
        cfg.precision = prec
        rep = SiReport()

        def call():
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            ctx.check(lib.si_spectral_init_device(ctx.ptr, C.byref(g), a.nc, a.seed, pts.data_ptr(), pts.shape[1],
                                                  C.byref(cfg), out.data_ptr(), C.byref(rep)))
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        for _ in range(max(1, min(a.warmup, 3))):
            call()
        sampler = ClockSampler(0) if prec == 1 else None
        if sampler:
            sampler.start()
        times = [call() for _ in range(a.steps)]
        if sampler:
            clocks = sampler.stop()
        results[name] = {"ms": statistics.mean(times), "ms_all": times, "components": rep.n_components_graph,
                         "iterations": rep.iterations, "level_max": rep.level, "max_residual": rep.max_residual}
    line = {"metric": "multi-component spectral init s (all components, residual<=1e-5)", "value":
            results["mixed"]["ms"] / 1e3, "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": results["mixed"]["ms"], "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 bulk + f64 Gram/RR/refinement", "data": "synthetic (seeded, built on the GPU)",
            "config": {"workload": f"{a.n_comp} disconnected fuzzy-kNN components, sizes log-uniform in [20, 100k], "
                                   "1-10 clusters in 20-D, k=15; full pipeline with spectral meta-embedding",
                       "n": n, "nnz": nnz, "size_max": int(sizes.max()), "size_min": int(sizes.min()),
                       "graph_build_s": round(t_gen, 1)},
            "fp64": results["fp64"], "mixed": results["mixed"], "clocks": clocks}
    print(json.dumps(line))


def run_configs(a):
    """One JSON line per parity configuration (device time per solve, CUDA events)."""
    import numpy as np
    import torch
    import spectral_init_b200 as si
    from spectral_init_b200 import synthetic
    from spectral_init_b200._lib import SiConfig, SiReport
    from spectral_init_b200.warm_start import WEIGHTS_PATH, DeviceLaplacian, WarmStartModel
    dev = torch.device("cuda", 0)
    ctx = si.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.si_ctx_stream(ctx.ptr), device=dev)
    model = None
    if WEIGHTS_PATH.exists():
        model = WarmStartModel.load(ctx=ctx)
        model.attach()

    def solve(lap, nc, prec=0, warm=0, level=-1, over=-1, nbiter=0, tol=0.0):
        cfg = SiConfig()
        lib.si_config_default(C.byref(cfg))
        cfg.precision, cfg.warm_start, cfg.force_level = prec, warm, level
        cfg.rsvd_oversampling, cfg.rsvd_nbiter = over, nbiter
        cfg.tol = tol
        k = nc + 1
        vals = (C.c_double * k)()
        vecs = torch.empty(lap.n, k, dtype=torch.float64, device=dev)
        lev = C.c_int32(-1)
        rep = SiReport()
        times = []
        for _ in range(max(1, a.warmup) + max(1, a.steps)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.si_solve_eigenproblem(ctx.ptr, C.byref(lap.op()), nc, a.seed, lap.sqrt_deg.data_ptr(),
                                                C.byref(cfg), vals, vecs.data_ptr(), C.byref(lev), C.byref(rep)))
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        times = times[max(1, a.warmup):]
        return {"ms": statistics.mean(times), "iterations": rep.iterations, "level": lev.value,
                "max_residual": rep.max_residual}, np.array(vals[:]), vecs

    def sin_theta(x, y):
        qa, _ = torch.linalg.qr(x)
        qb, _ = torch.linalg.qr(y)
        return float(torch.linalg.matrix_norm(qb - qa @ (qa.T @ qb), ord=2))

    # n = 200k family graph: plain FP64 vs mixed vs learned start
    n = 200_000
    x = synthetic.gaussian_mixture_gpu(n, 30, 50, 2024, 2.0, 0.02, anisotropic=True, dirichlet_alpha=0.5, device=dev)
    idx, dist = synthetic.knn_gpu(x, 15)
    del x
    sigma, rho = synthetic.smooth_knn_gpu(dist, 15)
    g = synthetic.fuzzy_graph_gpu(idx, dist, sigma, rho)
    del idx, dist
    lap = DeviceLaplacian((g[0], g[1], g[2], n), ctx=ctx)
    import argparse as _ap
    orc = None if a.no_oracle else host_oracle(_ap.Namespace(n=n), g[0], g[1], g[2], 3)
    r64, v64, x64 = solve(lap, 2)
    if orc is not None:
        r64["vs_oracle"] = oracle_errors(orc, v64, x64)
    line = {"config": "n=200k: 30 anisotropic clusters (Dirichlet 0.5 sizes) in 50-D + 2% background, k=15, "
                      "n_components=2", "nnz": lap.nnz, "fp64": r64,
            "oracle": None if orc is None else orc["summary"]}
    legs = [("mixed", 1, 0, 0.0), ("learned", 1, 1, 0.0), ("fp64_tol", 0, 0, a.tol), ("mixed_tol", 1, 0, a.tol),
            ("learned_tol", 1, 1, a.tol)]
    for name, prec, warm, tol in legs:
        if warm and model is None:
            continue
        r, v, xv = solve(lap, 2, prec, warm, tol=tol)
        r["tol"] = tol if tol > 0 else 1e-5
        r["eigenvalue_abs_diff_vs_fp64"] = float(np.max(np.abs(v - v64)))
        r["sin_theta_vs_fp64"] = sin_theta(xv[:, 1:], x64[:, 1:])
        r["speedup_vs_fp64"] = r64["ms"] / r["ms"]
        if orc is not None:
            r["vs_oracle"] = oracle_errors(orc, v, xv)
        line[name] = r
    line["eigengap_2_3"] = float(v64[2] - v64[1])
    print(json.dumps(line), flush=True)
    del lap, g

    # n = 1M, k = 30 (the large-graph configuration: 100-cluster mixture in 50-D + 5 % background, ~45M
    # stored entries): LOBPCG at n_components 2 and 8 (FP64 at the crate's tolerance, mixed at --tol), the
    # rSVD path (oversampling 10, 4 power iterations), and the SpMM bandwidth at 4- and 16-wide blocks
    import argparse as _ap
    a30 = _ap.Namespace(**vars(a))
    a30.k = 30
    ip, ix, dv = make_graph(a30, dev, 0)
    lap = DeviceLaplacian((ip, ix, dv, a30.n), ctx=ctx)
    line = {"config": workload_name(a30).replace(f"n_components={a.nc}", "n_components 2 and 8, LOBPCG and rSVD"),
            "nnz": lap.nnz}
    op = lap.op()
    plan = C.c_void_p()
    ctx.check(lib.si_operator_plan_create(ctx.ptr, C.byref(op), C.byref(plan)))
    peaks, peak_src = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    for ld in (4, 16):
        for f32 in (True, False):
            xb = 4 if f32 else 8
            x = torch.randn(a30.n, ld, dtype=torch.float32 if f32 else torch.float64, device=dev)
            y = torch.empty_like(x)
            fn = lib.si_spmm_planned_f32 if f32 else lib.si_spmm_planned
            for _ in range(3):
                ctx.check(fn(ctx.ptr, plan, x.data_ptr(), y.data_ptr(), ld))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(20):
                ctx.check(fn(ctx.ptr, plan, x.data_ptr(), y.data_ptr(), ld))
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / 20
            byt = lap.nnz * (4 + xb) + (a30.n + 1) * 8 + 2 * a30.n * ld * xb
            line[f"spmm_ld{ld}_{'f32' if f32 else 'f64'}"] = {"ms": ms, "gbs": byt / ms / 1e6,
                                                              "frac_of_hbm": byt / ms / 1e6 / hbm}
            del x, y
    lib.si_operator_plan_destroy(plan)
    line["hbm_peak_gbs"] = {"value": hbm, "source": peak_src}
    for nc in (2, 8):
        line[f"lobpcg_nc{nc}_fp64"], _, _ = solve(lap, nc)
        line[f"lobpcg_nc{nc}_mixed"], _, _ = solve(lap, nc, 1, tol=a.tol)
        line[f"rsvd_nc{nc}"], _, _ = solve(lap, nc, 0, 0, 4, 10, 4)
    print(json.dumps(line), flush=True)


def run_learned_eval(a):
    """Learned vs random warm start on held-out graphs of the benchmark family
    (n = --n, k = --k; the network was trained on n = 10k-200k graphs and never
    saw these), mixed precision at --tol, device time with CUDA events."""
    import argparse as _ap
    import torch
    import spectral_init_b200 as si
    from spectral_init_b200._lib import SiConfig, SiReport
    from spectral_init_b200.warm_start import WEIGHTS_PATH, DeviceLaplacian, WarmStartModel
    dev = torch.device("cuda", 0)
    ctx = si.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.si_ctx_stream(ctx.ptr), device=dev)
    if not WEIGHTS_PATH.exists():
        print(json.dumps({"learned_eval": True, "unavailable": "no trained weights"}))
        return
    model = WarmStartModel.load(ctx=ctx)
    model.attach()
    rows = []
    for g_i in range(a.learned_eval):
        ag = _ap.Namespace(**vars(a))
        ag.seed = a.seed + 1 + g_i
        ip, ix, dv = make_graph(ag, dev, 0)
        lap = DeviceLaplacian((ip, ix, dv, a.n), ctx=ctx)
        row = {"seed": ag.seed, "nnz": lap.nnz}
        for name, warm in (("random", 0), ("learned", 1)):
            cfg = SiConfig()
            lib.si_config_default(C.byref(cfg))
            cfg.precision = 1
            cfg.warm_start = warm
            cfg.tol = a.tol
            cfg.learned_filter = a.learned_filter
            cfg.mixed_switch_tol = a.switch_tol
            k = a.nc + 1
            vals = (C.c_double * k)()
            vecs = torch.empty(a.n, k, dtype=torch.float64, device=dev)
            lev = C.c_int32(-1)
            rep = SiReport()
            times = []
            for _ in range(2):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.check(lib.si_solve_eigenproblem(ctx.ptr, C.byref(lap.op()), a.nc, a.seed, lap.sqrt_deg.data_ptr(),
                                                    C.byref(cfg), vals, vecs.data_ptr(), C.byref(lev), C.byref(rep)))
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            row[name] = {"ms": times[-1], "iterations": rep.iterations, "fp32_iterations": rep.fp32_iterations,
                         "level": lev.value, "max_residual": rep.max_residual, "learned_start": rep.learned_start}
        rows.append(row)
        print(json.dumps(row), flush=True)
        del lap, ip, ix, dv
    model.close()
    it_l = statistics.mean(r["learned"]["iterations"] for r in rows)
    it_r = statistics.mean(r["random"]["iterations"] for r in rows)
    ms_l = statistics.mean(r["learned"]["ms"] for r in rows)
    ms_r = statistics.mean(r["random"]["ms"] for r in rows)
    print(json.dumps({"learned_eval": True, "workload": workload_name(a), "tol": a.tol, "graphs": len(rows),
                      "learned_filter": a.learned_filter,
                      "mean_iterations_learned": it_l, "mean_iterations_random": it_r, "mean_ms_learned": ms_l,
                      "mean_ms_random": ms_r, "rows": rows}))


def run_dense(a):
    """One JSON line: the device dense eigensolver (level 0) on fuzzy-kNN graphs of a few sizes, device time
    per solve with CUDA events on the library's stream."""
    import torch
    import spectral_init_b200 as si
    from spectral_init_b200 import synthetic
    from spectral_init_b200._lib import SiConfig, SiReport
    from spectral_init_b200.warm_start import DeviceLaplacian
    dev = torch.device("cuda", 0)
    ctx = si.Context(0)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(lib.si_ctx_stream(ctx.ptr), device=dev)
    out = {"config": "dense eigensolver (level 0), n_components=2: fuzzy-kNN graphs, 4-cluster Gaussian mixture "
                     "in 20-D (unit centre spread), k=15, seed 7", "sizes": {}}
    for n in (300, 1000, 1900):
        ip, ix, dv = synthetic.fuzzy_knn_graph_gpu(n, 15, 4, 20, seed=7, center_std=1.0, device=dev)
        lap = DeviceLaplacian((ip, ix, dv, n), ctx=ctx)
        cfg = SiConfig()
        lib.si_config_default(C.byref(cfg))
        cfg.force_level = 0
        vals = (C.c_double * 3)()
        vecs = torch.empty(n, 3, dtype=torch.float64, device=dev)
        lev = C.c_int32(-1)
        rep = SiReport()
        times = []
        for _ in range(max(1, a.warmup) + max(1, a.steps)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.si_solve_eigenproblem(ctx.ptr, C.byref(lap.op()), 2, a.seed, lap.sqrt_deg.data_ptr(),
                                                C.byref(cfg), vals, vecs.data_ptr(), C.byref(lev), C.byref(rep)))
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        times = times[max(1, a.warmup):]
        out["sizes"][str(n)] = {"ms": statistics.mean(times), "level": lev.value, "eigenvalues": list(vals[:]),
                                "max_residual": rep.max_residual}
    print(json.dumps(out), flush=True)


def main():
    a = parse_args()
    if a.cpu_only:
        run_cpu_only(a)
        return
    if a.components and a.impl == "ours":
        run_components(a)
        return
    if a.learned_eval and a.impl == "ours":
        run_learned_eval(a)
        return
    if a.dense and a.impl == "ours":
        run_dense(a)
        return
    if a.configs and a.impl == "ours":
        run_configs(a)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
