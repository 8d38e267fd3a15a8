#!/usr/bin/env python
"""Benchmark of the ART hot path on B200: batched weighted ridge solves.

Workload (one step): 65,536 independent weighted ridge systems, n_k
log-uniform in [64, 8192] (about 110M rows), x uniform on [-1,1]^d with
d in {8, 16}, affine or full quadratic features (p = 9, 17, 45, 153; a
quarter each), weights = products of 1-8 sigmoids, noisy random quadratic
y, ridge log-uniform in [1e-8, 1e-2]; seeded synthetic data generated on the
device.  The inputs (~12 GB) are larger than L2, so no flush is needed
between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank solves its own 65,536-system batch (weak scaling, no
data-path collective); rank 0 prints one JSON line with the max-over-ranks
device time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "ridge solves/s"
# DRAM bytes (read + write) per row of the tensor-core class, from the ncu
# capture of the tensor-core ridge kernel on the 8,192-system case at the
# tuned threshold (153 features): 1.0477 GB read + 0.0180 GB written over the
# class's 3,296,275 rows (the first pass reads x, y, w; the refinement passes
# re-read x and w).
RIDGE_TC_DRAM_BYTES_PER_ROW = 1.065706e9 / 3296275
UNIT = "solves/s"
WORKLOAD = ("batched weighted ridge: 65,536 systems/GPU, n log-uniform [64, 8192], d in {8,16}, "
            "affine or quadratic features (p = 9/17/45/153), sigmoid-product weights, "
            "ridge log-uniform [1e-8, 1e-2], solver normal")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--systems", type=int, default=65536)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--cpu-per-class", type=int, default=256,
                    help="systems per feature class in the timed CPU sample")
    ap.add_argument("--fp64-factor", action="store_true",
                    help="mixed form factors the tensor-core Gram in FP64")
    ap.add_argument("--variants", action="store_true",
                    help="also time the other mixed-form factorisation variant")
    ap.add_argument("--per-node-per-class", type=int, default=64,
                    help="systems per feature class in the per-node FP64 sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="skip the split-search and hit-and-run legs")
    ap.add_argument("--legs", default="split_level,hit_and_run,tree_build,serving",
                    help="comma-separated legs to run after the headline")
    ap.add_argument("--split-nodes", type=int, default=4096)
    ap.add_argument("--har-chains", type=int, default=16384)
    ap.add_argument("--tree-builds", type=int, default=2)
    ap.add_argument("--tree-cohort", type=int, default=256,
                    help="BFS cohort size (node_batch_size) of both tree-build forms")
    ap.add_argument("--serve-jobs", type=int, default=2000)
    ap.add_argument("--serve-seconds", type=float, default=30.0,
                    help="admission window of the serving stream (seconds of wall clock)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default launch shapes")
    ap.add_argument("--tensor-min-features", type=int, default=None,
                    help="fix the mixed form's tensor-core threshold instead of tuning it")
    ap.add_argument("--autotune-per-class", type=int, default=1024,
                    help="systems per feature class in the autotuner's sample")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"art_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_id_for(device_index: int) -> str:
    import torch

    try:
        uuid = str(torch.cuda.get_device_properties(device_index).uuid)
        return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        return vis.split(",")[device_index] if vis else str(device_index)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# B200 dense FP64 (vector and tensor), NVIDIA's published figure; the pool's
# measured peaks cover HBM and bf16 only, so FP64 fractions are "of spec".
FP64_SPEC_TFLOPS = 37.0


def cpu_split_rate(wl, nodes=4, restarts=16, iters=60, seed=0):
    """The oracle's projected-gradient loop (the reference's CPU split path)
    on a sample of the level's nodes: ``nodes`` nodes spaced in n, ``restarts``
    restarts each, the level's 60 annealed steps.  Returns restart-steps/s
    for the level's mean n (the CPU cost of a restart-step is linear in n:
    row-restart-steps/s divided by the mean rows per node), cores, the sample
    text and the seconds spent."""

    from threadpoolctl import threadpool_limits

    from oracle import ridge as O
    from oracle import split as S

    cores = len(os.sched_getaffinity(0))
    x = wl.x.cpu().numpy() if hasattr(wl.x, "cpu") else np.asarray(wl.x)
    y = wl.y.cpu().numpy() if hasattr(wl.y, "cpu") else np.asarray(wl.y)
    th0 = wl.theta0.cpu().numpy() if hasattr(wl.theta0, "cpu") else np.asarray(wl.theta0)
    n = np.diff(wl.row_offsets)
    order = np.argsort(n, kind="stable")
    pick = order[np.linspace(0, n.size - 1, nodes + 2).round().astype(int)[1:-1]]
    p = S.Params(max_iters=iters, n_restarts=restarts, grad_atol=0.0, grad_rtol=0.0, min_side_points=8,
                 min_side_fraction=0.0, anneal_ratio=0.1)
    rows_steps, t_all = 0.0, 0.0
    with threadpool_limits(limits=cores):
        for k in pick:
            r0, r1 = int(wl.row_offsets[k]), int(wl.row_offsets[k + 1])
            X = x[r0 * wl.d: r1 * wl.d].reshape(-1, wl.d)
            yy = y[r0:r1]
            t0 = time.perf_counter()
            for r in range(restarts):
                opt = S.optimize(X, yy, th0[k, r], float(wl.temperature[k]), O.AFFINE, float(wl.ridge[k]), p)
                rows_steps += (r1 - r0) * max(1, opt["n_iters"])
            t_all += time.perf_counter() - t0
    rate = rows_steps / t_all / float(n.mean())
    sample = (f"{nodes} nodes (n = {', '.join(str(int(n[k])) for k in pick)}) x {restarts} restarts x {iters} "
              f"annealed steps ({t_all:.1f} s), scaled to the level's mean n = {n.mean():.0f}")
    return rate, cores, sample, t_all


def cpu_har_rate(d, chains=1024, steps=1000, seed=4):
    """The oracle's batched chain transition (the reference's numba kernel
    restated in numpy, vectorised over chains) with host normal/uniform draws,
    on ``chains`` chains of the benchmark's polytope family for ``steps``
    steps.  Returns chain-steps/s, cores, sample text, seconds."""

    from threadpoolctl import threadpool_limits

    from oracle import sampling as H

    cores = len(os.sched_getaffinity(0))
    rng = np.random.default_rng([seed, d, 1])
    k = 8
    c = rng.uniform(-0.5, 0.5, d)
    Ao = rng.normal(size=(k, d))
    Ao /= np.linalg.norm(Ao, axis=1, keepdims=True)
    bo = Ao @ c + rng.uniform(0.05, 0.5, k)
    Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
    A, b = np.vstack([Ab, Ao]), np.concatenate([bb, bo])
    with threadpool_limits(limits=cores):
        t0 = time.perf_counter()
        dirs = rng.normal(size=(chains, steps, d))
        unif = rng.random(size=(chains, steps))
        H.chains_batched(A, b, np.repeat(c[None], chains, 0), dirs, unif, 0, 10, steps // 10)
        secs = time.perf_counter() - t0
    return chains * steps / secs, cores, (f"{chains} chains x {steps} steps in one polytope of the family "
                                          f"(box cut by {k} halfspaces), draws included ({secs:.1f} s)"), secs


def cpu_serving_rate(jobs, budget_s=20.0, n_max=20000):
    """The oracle's depth-first build, fixed-sample form (children keep their
    inherited samples, as the service does), of the stream's jobs in arrival
    order with n0 <= n_max, one at a time, until ``budget_s`` of CPU time:
    the job's target, leaf model, temperature, iteration cap, minimum side
    count, depth limit and 3 refinement rounds of +10% hit-and-run samples in
    the 4 leaves of largest error.  Returns builds/s, cores, sample text."""

    from threadpoolctl import threadpool_limits

    from art.serving import _target_numpy
    from oracle import builder as B
    from oracle import split as S

    cores = len(os.sched_getaffinity(0))
    done, rows, t_all = 0, 0, 0.0
    with threadpool_limits(limits=cores):
        for job in jobs:
            if job.n_initial > n_max:
                continue
            t0 = time.perf_counter()
            p = job.n_features
            b = B.Builder(-np.ones(job.dim), np.ones(job.dim), _target_numpy(job), job.kind, job.ridge,
                          job.temperature, job.error_threshold, job.max_depth, job.n_initial,
                          S.Params(max_iters=job.max_iters, n_restarts=1, grad_atol=1e-8, grad_rtol=1e-5,
                                   min_side_points=job.min_side_points or 2 * p, min_side_fraction=0.0),
                          burn_in=0, thinning=10, random_state=job.seed % (2**31), top_up=False,
                          refinement_rounds=job.rounds,
                          refinement_points=int(round(job.grow_fraction * job.n_initial)),
                          refinement_leaves=job.refine_leaves)
            b.build()
            t_all += time.perf_counter() - t0
            done += 1
            rows += job.n_final
            if t_all > budget_s:
                break
    return done / t_all, cores, (f"{done} jobs of the stream with n0 <= {n_max} (mean {rows / max(done, 1):.0f} "
                                 f"final rows), built one at a time ({t_all:.1f} s)")


def cpu_tree_rate(f, builds=1, **kw):
    """The oracle's depth-first build (pinned to the reference's trees) of the
    tree configuration, with the same refinement driver.  Returns builds/s,
    cores, sample text, seconds."""

    from threadpoolctl import threadpool_limits

    from oracle import builder as B
    from oracle import ridge as O
    from oracle import split as S

    cores = len(os.sched_getaffinity(0))
    with threadpool_limits(limits=cores):
        t0 = time.perf_counter()
        for _ in range(builds):
            b = B.Builder(-np.ones(2), np.ones(2), f, O.AFFINE, 1e-6, 0.05, 0.02, 6, 4096,
                          S.Params(max_iters=100, n_restarts=1, min_side_points=32, min_side_fraction=0.0),
                          burn_in=0, thinning=5, random_state=1, **kw)
            root = b.build()
        secs = time.perf_counter() - t0
    nodes = sum(1 for _ in B.iter_nodes(root))
    return builds / secs, cores, f"{builds} build(s), {nodes} nodes, depth-first ({secs:.1f} s)", secs


def algorithmic(wl, idx=None):
    """Algorithmic work per system: F = n p(p+1) + 2np + p^3/3 + 2p^2 flops; B = n (d+2) 8 + 8p bytes."""

    from art.models import kind_feature_count

    n = np.diff(wl.row_offsets).astype(float)
    d = wl.dims.astype(float)
    p = np.array([kind_feature_count(int(a), int(b)) for a, b in zip(wl.dims, wl.kinds)], float)
    if idx is not None:
        n, d, p = n[idx], d[idx], p[idx]
    flops = n * p * (p + 1) + 2 * n * p + p ** 3 / 3 + 2 * p ** 2
    nbytes = n * (d + 2) * 8 + 8 * p
    return float(flops.sum()), float(nbytes.sum())


def stratified_sample(wl, per_class: int, seed: int = 0):
    """Systems evenly spaced in n within each (d, kind) class."""

    idx = []
    n = np.diff(wl.row_offsets)
    for key in sorted(set(zip(wl.dims.tolist(), wl.kinds.tolist()))):
        members = np.flatnonzero((wl.dims == key[0]) & (wl.kinds == key[1]))
        order = members[np.argsort(n[members], kind="stable")]
        take = np.linspace(0, order.size - 1, min(per_class, order.size)).round().astype(int)
        idx.append(order[take])
    return np.concatenate(idx)


def cpu_solve_rate(wl, per_class, repeats: int = 1, mix=None):
    """Time the oracle (reference CPU algorithm) on a stratified sample; scale to the mix.

    ``per_class=None`` means ``wl`` already is the sample and ``mix`` holds
    the class counts of the full workload.
    """

    from oracle import ridge as O
    from threadpoolctl import threadpool_limits

    cores = len(os.sched_getaffinity(0))
    if per_class is None:
        sample = np.arange(wl.count)
        sub = wl
    else:
        sample = stratified_sample(wl, per_class)
        sub = wl.subset(sample)
        mix = {key: int(np.sum((wl.dims == key[0]) & (wl.kinds == key[1])))
               for key in set(zip(wl.dims.tolist(), wl.kinds.tolist()))}
    per_class_time = {}
    t_all = 0.0
    with threadpool_limits(limits=cores):
        for _ in range(repeats):
            for k in range(sub.count):
                r0, r1 = sub.row_offsets[k], sub.row_offsets[k + 1]
                d = int(sub.dims[k])
                X = sub.x[sub.x_offsets[k]: sub.x_offsets[k] + (r1 - r0) * d].reshape(-1, d)
                t0 = time.perf_counter()
                phi = O.features(X, int(sub.kinds[k]))
                try:
                    O.solve_weighted_ridge(phi, sub.y[r0:r1], sub.w[r0:r1], float(sub.ridge[k]), solver="normal")
                except np.linalg.LinAlgError:
                    pass
                dt = time.perf_counter() - t0
                key = (int(sub.dims[k]), int(sub.kinds[k]))
                per_class_time.setdefault(key, []).append(dt)
                t_all += dt
    est = 0.0
    total = 0
    for key, ts in per_class_time.items():
        est += mix[key] * float(np.mean(ts))
        total += mix[key]
    rate = total / est
    return rate, cores, sample.size, t_all


# ------------------------------------------------------------------ arms
def run_reference(args):
    """--impl reference: the reference CPU algorithm (oracle port) on the host cores."""

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl, mix = _cpu_workload(args.systems, args.cpu_per_class)
    times, walls = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rate, cores, sample, _ = cpu_solve_rate(wl, None, mix=mix)
        if i >= args.warmup:
            times.append(rate)
            walls.append(time.perf_counter() - t0)
    value = float(np.median(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        # one step = the timed sample; the full 65,536-system workload would take
        # ms_per_full_workload (extrapolated from the sample's per-class times)
        "ms_per_step": 1000.0 * float(np.mean(walls)),
        "ms_per_full_workload": 1000.0 * args.systems / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "systems": args.systems, "solver": "normal"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{sample} systems stratified by n in each of 4 feature classes, scaled to the mix"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _cpu_workload(systems, per_class):
    """The stratified sample of the benchmark's systems with numpy-drawn rows.

    Per-system parameters (n, d, features, ridge, weights, target) are the
    device workload's own; only the row values come from numpy.  Returns the
    sample and the class counts of the full mix.
    """

    from art import workloads

    meta = workloads.ridge_systems(systems, seed=2, device=None, only=[])
    full = _Meta(meta)
    sample = stratified_sample(full, per_class)
    wl = workloads.ridge_systems(systems, seed=2, device=None, only=sample)
    return wl, full.class_counts()


class _Meta:
    """Per-system sizes of the full mix without rows."""

    def __init__(self, empty_wl):
        from art import workloads

        rng_meta = workloads.ridge_meta(empty_wl)
        self.row_offsets, self.dims, self.kinds = rng_meta

    @property
    def count(self):
        return int(self.dims.shape[0])

    def class_counts(self):
        keys, counts = np.unique(np.stack([self.dims, self.kinds], 1), axis=0, return_counts=True)
        return {(int(a), int(b)): int(c) for (a, b), c in zip(keys, counts)}


def per_node_rate(args, wl, ro, xo, dims, kinds, ridge, out, stream):
    """Plain FP64 form called once per system (count 1 per C-ABI call, no
    batching), on a stratified sample; the per-system device time is averaged
    over the sample with the workload's class mix and reported as solves/s."""

    import ctypes as C

    import torch

    from art import _native as N

    lib = N.load_library()
    idx = stratified_sample(wl, args.per_node_per_class)
    x, y, w = wl.x, wl.y, wl.w
    P = int(out.beta.shape[1])
    ws = torch.empty(lib.art_ridge_workspace_size(1, P), dtype=torch.uint8, device=x.device)
    h = C.c_void_p(stream.cuda_stream)

    def addr(t, k):
        return C.c_void_p(t.data_ptr() + k * t.element_size() * (t.shape[1] if t.dim() == 2 else 1))

    def call(k):
        seg = N.ArtSegments(1, addr(ro, k), addr(xo, k), addr(dims, k), addr(kinds, k))
        prob = N.ArtRidgeProblem(seg, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(w.data_ptr()),
                                 addr(ridge, k), 1e-12, N.SOLVER_NORMAL, N.PRECISION_FP64, 1e-10, P,
                                 int(wl.max_dim), 0, 0)
        res = N.ArtRidgeResult(addr(out.beta, k), P, addr(out.ridge_effective, k), None, addr(out.status, k),
                               addr(out.info, k))
        N.check(lib.art_ridge_batched(C.byref(prob), C.byref(res), C.c_void_p(ws.data_ptr()), ws.numel(), h),
                "art_ridge_batched")

    for k in idx[:8]:
        call(int(k))
    torch.cuda.synchronize()
    cls = list(zip(wl.dims[idx].tolist(), wl.kinds[idx].tolist()))
    per_cls = {}
    for k, key in zip(idx, cls):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        call(int(k))
        e1.record(stream)
        per_cls.setdefault(key, []).append((e0, e1))
    torch.cuda.synchronize()
    mix = {key: int(np.sum((wl.dims == key[0]) & (wl.kinds == key[1]))) for key in per_cls}
    total = sum(mix.values())
    avg_ms = sum(mix[key] / total * np.mean([a.elapsed_time(b) for a, b in evs]) for key, evs in per_cls.items())
    return {"value": 1000.0 / avg_ms, "unit": UNIT, "sample": f"{len(idx)} systems stratified by n over the "
            f"feature classes, one art_ridge_batched call each, scaled to the class mix",
            "ms_per_system": avg_ms}


def _event_ms(fn, steps, warmup, stream):
    import torch

    out = None
    for _ in range(warmup):
        out = fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, out


def leg_split(args, stream):
    """Batched soft oblique split search: 4096 nodes, d = 16, n log-uniform in
    [256, 16384], 16 restarts x 60 projected-gradient steps, affine child fits
    (lambda = 1e-6), temperature annealed 0.2 -> 0.02; the plain FP64 form
    and the mixed form (single-precision gates, FP64 sums and solves) in the
    tuned launch form (one warp per restart unless a CTA shape timed faster),
    the FP64 CTA form at its best tuned shape, and the mixed CTA form with
    the tensor-core Gram."""

    from art import _native as N
    from art import autotune
    from art import workloads
    from art.models import AffineRidgeModel
    from art.splitters import SoftObliqueSplitter, split_level

    wl = workloads.split_nodes(args.split_nodes, device="cuda")
    sp = SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 0.2, max_iters=60, grad_atol=0.0, grad_rtol=0.0,
                             min_side_points=8, min_side_fraction=0.0, n_restarts=16)
    # launch shape tuned on a separate 296-node level of the same distribution
    tw = workloads.split_nodes(296, seed=33, device="cuda")
    tuned = autotune.tune_split_shape(sp, tw.x, tw.y, tw.row_offsets, tw.dims, tw.kinds, tw.temperature, tw.ridge,
                                      max_dim=tw.d, max_features=tw.d + 1, theta0=tw.theta0, anneal_ratio=0.1,
                                      repeats=1, stream=stream) if not args.no_autotune else None
    units = wl.count * 16 * 60
    n = np.diff(wl.row_offsets).astype(float)
    d, p, H = wl.d, wl.d + 1, 4
    flops = float((n * (2 * d + p * (p + 1) + 8 * p + 2 * d + 12 + 6 * H)).sum()) * 16 * 60
    out = {"metric": "split restart-steps/s", "unit": "restart-steps/s", "nodes": wl.count, "rows": wl.n_rows,
           "restarts": 16, "iterations": 60, "autotune": tuned}
    thetas = {}
    # best CTA-form shape among the tuned candidates (keys g x h x c x w)
    cta_shape = (4, 2, 1, 0)
    if tuned:
        cta = {k: v for k, v in tuned["candidates_ms"].items() if k.endswith("x0")}
        if cta:
            cta_shape = tuple(int(v) for v in min(cta, key=cta.get).split("x"))
    out["cta_shape"] = list(cta_shape)
    variants = (("fp64", "fp64", False, None), ("mixed", "mixed", False, None), ("fp64_cta", "fp64", False, cta_shape),
                ("mixed_tc", "mixed", True, (0, 0, 0, 0)))
    for prec, precision, tensor, shape in variants:
        sp.precision = precision
        sp.tensor_gram = tensor
        kw = {} if shape is None else dict(group_restarts=shape[0], trial_steps=shape[1], ctas_per_sm=shape[2],
                                           restart_warps=shape[3])

        def step():
            return split_level(sp, wl.x, wl.y, wl.row_offsets, wl.dims, wl.kinds, wl.temperature, wl.ridge,
                               theta0=wl.theta0, anneal_ratio=0.1, hard_refit=True, max_dim=wl.d,
                               max_features=wl.d + 1, stream=stream, **kw)

        N.profile_reset()
        N.profile_enable(True)
        ms, res = _event_ms(step, 1, 1, stream)
        N.profile_enable(False)
        prof = N.profile_report()
        top = max(prof.items(), key=lambda kv: kv[1][1])
        thetas[prec] = (res.loss.cpu().numpy(), res.n_right.cpu().numpy())
        out[prec] = {"value": units / (ms / 1000.0), "ms_per_step": ms,
                     "mean_iters_chosen": float(res.n_iters.double().mean().item()),
                     "failures": int((res.failure != 0).sum().item()),
                     "achieved_fp64_tflops": flops / (ms / 1000.0) / 1e12, "kernel": top[0],
                     "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}
    hbm, bf16, peak_kind = peaks()
    for prec in ("fp64", "mixed", "fp64_cta", "mixed_tc"):
        kern = out[prec]["kernels"].get("split_level")
        if kern:
            kms = kern["ms"] / max(kern["launches"], 1)
            bytes_alg = float(n.sum()) * (d + 1) * 8 * 60          # x and y once per node-step, shared by restarts
            out[prec]["roofline"] = {
                "bound": "fp64", "kernel": "split_level", "achieved": flops / (kms / 1000.0) / 1e12,
                "peak": FP64_SPEC_TFLOPS, "unit": "TFLOP/s",
                "frac": flops / (kms / 1000.0) / 1e12 / FP64_SPEC_TFLOPS,
                "peak_source": "B200 FP64 spec sheet (no measured FP64 peak on this pool)",
                "algorithmic_bytes": bytes_alg, "achieved_gbs": bytes_alg / (kms / 1000.0) / 1e9,
                "hbm_frac": bytes_alg / (kms / 1000.0) / 1e9 / hbm, "hbm_peak_source": peak_kind,
                "launch_ms": kms}
    if not args.no_cpu:
        rate, cores, sample, secs = cpu_split_rate(wl)
        out["cpu_baseline"] = {"value": rate, "unit": "restart-steps/s", "cores": cores, "kind": "port",
                               "sample": sample}
        out["speedup_vs_cpu_fp64"] = out["fp64"]["value"] / rate
        out["speedup_vs_cpu_mixed"] = out["mixed"]["value"] / rate
    la, lb = thetas["fp64"][0], thetas["mixed"][0]
    ok = np.isfinite(la) & np.isfinite(lb)
    out["value"] = out["fp64"]["value"]
    out["mixed_speedup"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed_tc_speedup"] = out["fp64"]["ms_per_step"] / out["mixed_tc"]["ms_per_step"]
    out["warp_form_speedup_vs_cta_form"] = out["fp64_cta"]["ms_per_step"] / out["fp64"]["ms_per_step"]
    out["mixed_vs_fp64_hard_loss_rel_diff_median"] = float(np.median(np.abs(lb[ok] - la[ok]) / np.abs(la[ok])))
    out["mixed_same_partition_fraction"] = float(np.mean(thetas["fp64"][1] == thetas["mixed"][1]))
    return out


def leg_har(args, stream):
    """Batched hit-and-run: 16,384 chains, one polytope each (box [-1,1]^d cut
    by 4-12 oblique halfspaces), 2000 steps, thinning 10, device Philox draws,
    FP64 chords; d in {8, 16, 32, 64}."""

    from art import workloads
    from art.sampling import DevicePolytopes, hit_and_run_device

    out = {}
    for d in (8, 16, 32, 64):
        wl = workloads.polytopes(args.har_chains, d=d, device="cuda")
        polys = DevicePolytopes(d, wl.lo, wl.hi, wl.row_offsets, wl.A, wl.b, wl.max_rows)

        def step():
            return hit_and_run_device(polys, wl.chain_polytope, wl.x0, burn_in=0, thinning=10, n_rounds=200,
                                      seeds=wl.seeds, stream=stream)

        ms, (samples, x, status) = _event_ms(step, 1, 1, stream)
        steps = args.har_chains * 2000
        k_mean = float((wl.row_offsets[1:] - wl.row_offsets[:-1]).double().mean().item())
        flops = steps * (2 * k_mean * d + 7 * d + 6 * (2 * d + k_mean))
        hbm, _, peak_kind = peaks()
        bytes_alg = args.har_chains * 200 * d * 8 + int(wl.A.numel() + wl.b.numel() + 2 * wl.lo.numel()) * 8
        out[f"d{d}"] = {"value": steps / (ms / 1000.0), "unit": "chain-steps/s", "ms": ms,
                        "samples_per_s": args.har_chains * 200 / (ms / 1000.0),
                        "achieved_fp64_gflops": flops / (ms / 1000.0) / 1e9,
                        "status_ok": bool((status == 0).all().item()),
                        "roofline": {"bound": "fp64", "achieved": flops / (ms / 1000.0) / 1e12,
                                     "peak": FP64_SPEC_TFLOPS, "unit": "TFLOP/s",
                                     "frac": flops / (ms / 1000.0) / 1e12 / FP64_SPEC_TFLOPS,
                                     "peak_source": "B200 FP64 spec sheet (no measured FP64 peak on this pool)",
                                     "algorithmic_bytes": bytes_alg,
                                     "hbm_frac": bytes_alg / (ms / 1000.0) / 1e9 / hbm, "hbm_peak_source": peak_kind}}
        if not args.no_cpu:
            rate, cores, sample, _ = cpu_har_rate(d)
            out[f"d{d}"]["cpu_baseline"] = {"value": rate, "unit": "chain-steps/s", "cores": cores, "kind": "port",
                                            "sample": sample}
            out[f"d{d}"]["speedup_vs_cpu"] = out[f"d{d}"]["value"] / rate
    return {"metric": "hit-and-run chain-steps/s", "chains": args.har_chains, "steps": 2000, "thinning": 10,
            "by_dim": out}


def leg_serving(args, stream):
    """Surrogate-build service on the stream of 2,000 jobs: Poisson arrivals at
    20 jobs/s, d uniform over {2, 4, 8, 16, 32}, n0 log-uniform in [1e3, 1e6],
    depth <= 12, quadratic leaves for d <= 8 else affine, 3 adaptive rounds of
    +10% samples.  Jobs are admitted against the wall clock for
    ``--serve-seconds``; the admitted jobs then finish and the rest of the
    stream is reported as unserved (``backlog``: those that had arrived).
    Latency is arrival to completion.  Mixed and plain FP64 leaf fits; each
    precision first builds, untimed, the smallest job of each dimension in
    the stream.  The CPU baseline is the oracle's depth-first build of the
    first jobs of the stream (fixed-sample form, one job at a time)."""

    from art.serving import ServingEngine, SurrogateJob, poisson_jobs

    out = {}
    for precision in ("mixed", "fp64"):
        jobs = poisson_jobs(args.serve_jobs, 20.0, seed=5)
        # untimed warm-up in this precision: the smallest job of each
        # dimension in the stream, all admitted at once (first launches of
        # every kernel form the stream uses happen here, not in the timed run)
        warm = {}
        for j in jobs:
            if j.dim not in warm or j.n_initial < warm[j.dim].n_initial:
                warm[j.dim] = j
        ServingEngine(precision=precision, stream=stream).run(
            [SurrogateJob(**{**j.__dict__, "arrival": 0.0}) for j in warm.values()])
        eng = ServingEngine(precision=precision, stream=stream)
        t0 = time.perf_counter()
        res = eng.run(jobs, admit_until=args.serve_seconds)
        wall = time.perf_counter() - t0
        lat = np.array([r.latency for r in res]) if res else np.array([np.nan])
        out[precision] = {"jobs_completed": len(res), "builds_per_s": len(res) / wall, "wall_s": wall,
                          "p50_latency_s": float(np.percentile(lat, 50)),
                          "p99_latency_s": float(np.percentile(lat, 99)),
                          "backlog": eng.backlog, "unserved": eng.unserved,
                          "ticks": eng.ticks, "peak_active": eng.peak_active,
                          "rows_total": int(sum(r.n_rows for r in res))}
    out["mixed_vs_fp64_builds_per_s"] = out["mixed"]["builds_per_s"] / max(out["fp64"]["builds_per_s"], 1e-300)
    if not args.no_cpu:
        rate, cores, sample = cpu_serving_rate(poisson_jobs(args.serve_jobs, 20.0, seed=5))
        out["cpu_baseline"] = {"value": rate, "unit": "builds/s", "cores": cores, "kind": "port", "sample": sample}
    return {"metric": "surrogate builds/s and build latency",
            "stream": f"{args.serve_jobs} jobs at 20 jobs/s (seed 5), admission open for {args.serve_seconds} s",
            **out}


def leg_tree(args, stream):
    """Tree builds/s on the 2-d configuration: N = 4096 points per node,
    depth <= 6, min 32 points per side, soft oblique splits (T = 0.05, 100
    iterations), affine leaves (lambda = 1e-6), children topped up by
    hit-and-run with device Philox draws, then 2 refinement rounds of 1024
    new points in the 4 leaves of largest fit error.  Two GPU forms with the
    same random stream and the same BFS cohorts of up to ``--tree-cohort``
    nodes (so the same tree): the level-batched build (one split launch, one
    top-up launch and one mixed-form fit with FP64 refinement per cohort, CUDA
    graphs) against the plain FP64 per-node build (one split call, one top-up
    and one FP64 fit per node); held-out RMSE of each on
    20,000 uniform points.  The CPU baseline is the oracle's depth-first
    build (the reference's trees) with the same refinement driver."""

    from art import _native as N
    from art import (AffineRidgeModel, BoxDomain, HitAndRunSampler, RegressionTreeBuilder, SoftObliqueSplitter,
                     TemperatureConfig)
    from art.workloads import bumps_ridge_2d

    f = bumps_ridge_2d(1)
    X_test = np.random.default_rng(99).uniform(-1.0, 1.0, (20000, 2))
    y_test = f(X_test)

    def build(batched):
        model = AffineRidgeModel(ridge=1e-6, solver="normal")
        sp = SoftObliqueSplitter(model, 0.05, max_iters=100, min_side_points=32, min_side_fraction=0.0)
        b = RegressionTreeBuilder(domain=BoxDomain.hypercube(2, -1.0, 1.0), oracle=f, model_template=model,
                                  splitter=sp, error_threshold=0.01, max_depth=6, sample_count=4096,
                                  temperature_config=TemperatureConfig(strategy="splitter"), random_state=1,
                                  oracle_vectorized=True, traversal="bfs", level_dispatch=batched,
                                  batched_fits=batched, cohort_top_up=batched, cuda_graphs=batched,
                                  fit_precision="mixed" if batched else "fp64", isotropic_sampling=False,
                                  refinement_rounds=2, refinement_points=1024, refinement_leaves=4,
                                  node_batch_size=args.tree_cohort,
                                  sampler=HitAndRunSampler(burn_in=0, thinning=5, rng_mode="device"))
        return b.build()

    out = {}
    trees = {}
    for name, batched in (("level_batched_mixed", True), ("plain_fp64_per_node", False)):
        build(batched)  # warm-up (graph capture, autotune tables)
        torch_sync()
        N.profile_reset()
        N.profile_enable(True)
        t0 = time.perf_counter()
        reps = args.tree_builds
        for _ in range(reps):
            res = build(batched)
        torch_sync()
        wall = time.perf_counter() - t0
        N.profile_enable(False)
        prof = N.profile_report()
        kern_ms = sum(v[1] for v in prof.values())
        top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else ("none", (0, 0.0))
        rmse = float(np.sqrt(np.mean((res.tree.predict(X_test) - y_test) ** 2)))
        trees[name] = res
        out[name] = {"builds_per_s": reps / wall, "ms_per_build": 1000 * wall / reps,
                     "nodes": len(list(res.tree.iter_nodes())), "oracle_queries": res.oracle_queries,
                     "heldout_rmse": rmse, "gpu_kernel_ms_per_build": kern_ms / reps,
                     "gpu_busy_fraction": kern_ms / (1000 * wall),
                     "top_kernel": {"name": top[0], "launches_per_build": top[1][0] / reps,
                                    "ms_per_build": top[1][1] / reps}}
    out["speedup"] = out["level_batched_mixed"]["builds_per_s"] / out["plain_fp64_per_node"]["builds_per_s"]
    a, b = out["level_batched_mixed"]["heldout_rmse"], out["plain_fp64_per_node"]["heldout_rmse"]
    out["heldout_rmse_rel_diff"] = abs(a - b) / max(abs(b), 1e-300)
    ids = [[n.node_id for n in trees[k].tree.iter_nodes()] for k in trees]
    out["same_tree"] = ids[0] == ids[1]
    out["cohort"] = args.tree_cohort
    out["roofline"] = {"bound": "latency", "kernel": out["level_batched_mixed"]["top_kernel"]["name"],
                       "gpu_busy_fraction": out["level_batched_mixed"]["gpu_busy_fraction"],
                       "note": "hit-and-run top-ups are one chain per child, about 10^4 dependent steps each, so "
                               "a top-up launch lasts as long as its longest chain whatever the cohort size"}
    if not args.no_cpu:
        rate, cores, sample, _ = cpu_tree_rate(f, refinement_rounds=2, refinement_points=1024,
                                               refinement_leaves=4)
        out["cpu_baseline"] = {"value": rate, "unit": "builds/s", "cores": cores, "kind": "port", "sample": sample}
        out["speedup_vs_cpu"] = out["level_batched_mixed"]["builds_per_s"] / rate
    return {"metric": "tree builds/s", "sampler": "hit-and-run, device Philox draws", **out}


def torch_sync():
    import torch

    torch.cuda.synchronize()


def run_b200(args):
    import torch
    import torch.distributed as dist

    from art import _native as N
    from art import workloads
    from art.models import solve_weighted_ridge_batched

    from art.sharding import max_over_ranks, rank_info, rank_seed

    ri = rank_info()
    world, rank, local = ri.world, ri.rank, ri.local
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N.load_library()
    wl = workloads.ridge_systems(args.systems, seed=rank_seed(2, rank), device="cuda")
    ro = torch.from_numpy(wl.row_offsets).to(dev)
    xo = torch.from_numpy(wl.x_offsets).to(dev)
    dims = torch.from_numpy(wl.dims).to(dev)
    kinds = torch.from_numpy(wl.kinds).to(dev)
    ridge = torch.from_numpy(wl.ridge).to(dev)
    stream = torch.cuda.current_stream()

    def solve(precision, out=None, fp64_factor=None):
        return solve_weighted_ridge_batched(
            wl.x, wl.y, wl.w, ro, dims, kinds, ridge, x_offsets=xo, precision=precision,
            max_features=wl.max_features, max_dim=wl.max_dim, out=out,
            fp64_factor=(True if args.fp64_factor else None) if fp64_factor is None else fp64_factor,
            tensor_min_features=args.tensor_min_features)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(precision, fp64_factor=None):
        out = None
        for _ in range(args.warmup):
            out = solve(precision, out, fp64_factor)
        barrier()
        N.profile_reset()
        N.profile_enable(True)
        launches0 = N.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            out = solve(precision, out, fp64_factor)
        e1.record(stream)
        barrier()
        N.profile_enable(False)
        ms = e0.elapsed_time(e1)
        launches = N.launch_count() - launches0
        prof = N.profile_report()
        ms = max_over_ranks(ms)
        return ms / args.steps, launches // args.steps, prof, out

    # launch-shape choice of the mixed form, measured on a sample of this
    # batch before any timed region (the solves below read the tuned value)
    from art import autotune

    tuned = None
    if args.precision == "mixed" and not args.no_autotune and args.tensor_min_features is None:
        tuned = autotune.tune_ridge_threshold(wl.x, wl.y, wl.w, ro, dims, kinds, ridge, x_offsets=xo,
                                              max_dim=wl.max_dim, fp64_factor=True if args.fp64_factor else None,
                                              per_class=args.autotune_per_class, stream=stream)

    # plain FP64 form, batched and per node (one call per system, the
    # comparison point of the >=5x target), then the headline form
    plain_ms, _, plain_prof, plain_out = timed("fp64")
    per_node = (per_node_rate(args, wl, ro, xo, dims, kinds, ridge, plain_out, stream)
                if args.per_node_per_class > 0 else None)
    variants = {}
    if args.variants and args.precision == "mixed":
        v_ms, _, v_prof, v_out = timed("mixed", not args.fp64_factor)
        v_info = v_out.info.cpu().numpy()
        variants["fp64_factor" if not args.fp64_factor else "fp32_factor"] = {
            "ms_per_step": v_ms, "resolve_fraction": float(np.mean((v_info & N.INFO_FP64_RESOLVE) != 0)),
            "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in v_prof.items()}}
    with Clocks(gpu_id_for(local)) as clocks:
        ms, launches, prof, out = timed(args.precision)
    clk = clocks.summary()
    status = out.status.cpu().numpy()
    info = out.info.cpu().numpy()
    value = world * args.systems / (ms / 1000.0)

    # roofline of the dominant kernel
    hbm, bf16, peak_kind = peaks()
    top = max(prof.items(), key=lambda kv: kv[1][1])
    name, (n_launch, total_ms) = top
    per_launch_ms = total_ms / max(n_launch, 1)
    from art.models import kind_feature_count

    p_all = np.array([kind_feature_count(int(a), int(b)) for a, b in zip(wl.dims, wl.kinds)])
    if name == "ridge_warp":
        cls_idx = np.flatnonzero(p_all + 1 <= 24)
    elif "fp64<4>" in name:
        cls_idx = np.flatnonzero((p_all + 1 > 24) & (p_all + 1 <= 48) & ((p_all < 33) | (args.precision == "fp64")))
    elif "fp64<8>" in name:
        cls_idx = np.flatnonzero(p_all + 1 > 48) if args.precision == "fp64" else np.flatnonzero(info & N.INFO_FP64_RESOLVE)
    else:
        thr = args.tensor_min_features or (tuned["tensor_min_features"] if tuned else 33)
        cls_idx = np.flatnonzero(p_all >= thr)
    flops, nbytes = algorithmic(wl, cls_idx)
    achieved_gbs = nbytes / (per_launch_ms / 1000.0) / 1e9
    achieved_tf = flops / (per_launch_ms / 1000.0) / 1e12
    share = total_ms / sum(v[1] for v in prof.values())
    if name.startswith("ridge_tc"):
        # quadratic systems: 27-166 algorithmic flop/B, tensor-core bound;
        # traffic per launch from the ncu capture of the 8,192-system case
        # (DRAM bytes per tensor-class row, times this launch's rows)
        n_rows = float(np.diff(wl.row_offsets)[cls_idx].sum())
        roofline = {"bound": "tensor", "kernel": name, "achieved": achieved_tf, "peak": bf16,
                    "unit": "TFLOP/s", "frac": achieved_tf / bf16,
                    "traffic": RIDGE_TC_DRAM_BYTES_PER_ROW * n_rows if RIDGE_TC_DRAM_BYTES_PER_ROW else None,
                    "peak_source": f"{peak_kind} bf16 dense (the kernel issues TF32 hi/lo split products)",
                    "algorithmic_bytes": nbytes, "achieved_gbs": achieved_gbs, "hbm_frac": achieved_gbs / hbm,
                    "launch_ms": per_launch_ms, "kernel_share": share}
    else:
        roofline = {"bound": "hbm", "kernel": name, "achieved": achieved_gbs, "peak": hbm,
                    "unit": "GB/s", "frac": achieved_gbs / hbm, "traffic": None, "peak_source": peak_kind,
                    "achieved_tflops": achieved_tf, "launch_ms": per_launch_ms, "kernel_share": share}

    # end-to-end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        hx = torch.empty(wl.x.shape, dtype=torch.float64, pin_memory=True)
        hy = torch.empty(wl.y.shape, dtype=torch.float64, pin_memory=True)
        hw = torch.empty(wl.w.shape, dtype=torch.float64, pin_memory=True)
        hx.copy_(wl.x); hy.copy_(wl.y); hw.copy_(wl.w)
        meta = [torch.from_numpy(a).pin_memory() for a in (wl.row_offsets, wl.x_offsets, wl.dims, wl.kinds, wl.ridge)]
        hbeta = torch.empty((args.systems, wl.max_features), dtype=torch.float64, pin_memory=True)
        hstat = torch.empty(args.systems, dtype=torch.int32, pin_memory=True)

        def e2e_step():
            o = solve_weighted_ridge_batched(hx, hy, hw, meta[0], meta[2], meta[3], meta[4], x_offsets=meta[1],
                                             precision=args.precision, max_features=wl.max_features,
                                             max_dim=wl.max_dim)
            hbeta.copy_(o.beta, non_blocking=True)
            hstat.copy_(o.status, non_blocking=True)

        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        barrier()
        e2e_ms = max(e0.elapsed_time(e1), 1000.0 * (time.perf_counter() - t0)) / args.steps
        e2e_ms = max_over_ranks(e2e_ms)
        h2d = sum(int(t.numel() * t.element_size()) for t in (hx, hy, hw, *meta))
        d2h = int(hbeta.numel() * 8 + hstat.numel() * 4)
        e2e = {"value": world * args.systems / (e2e_ms / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms}
        del hx, hy, hw

    legs = {}
    if rank == 0 and not args.no_legs:
        chosen = set(args.legs.split(","))
        for name, fn in (("split_level", leg_split), ("hit_and_run", leg_har), ("tree_build", leg_tree),
                         ("serving", leg_serving)):
            if name not in chosen:
                continue
            try:
                legs[name] = fn(args, stream)
            except Exception as exc:  # a failing leg is reported, the headline stands
                legs[name] = {"error": f"{type(exc).__name__}: {exc}"}

    cpu = None
    if rank == 0 and not args.no_cpu:
        # the same systems the GPU solved: a stratified sample copied to the host
        sample_idx = stratified_sample(wl, args.cpu_per_class)
        mix = {key: int(np.sum((wl.dims == key[0]) & (wl.kinds == key[1])))
               for key in set(zip(wl.dims.tolist(), wl.kinds.tolist()))}
        rate, cores, sample, secs = cpu_solve_rate(wl.subset(sample_idx), None, mix=mix)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{sample} systems stratified by n over the 4 feature classes "
                         f"({secs:.1f} s of CPU work), scaled to the 65,536-system mix"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    ok = float(np.mean(status == 0))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "tf32x3+f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "systems_per_gpu": args.systems, "precision": args.precision,
                   "rows_per_gpu": wl.n_rows, "l2": "inputs (~12 GB) larger than L2; no flush",
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "plain_fp64": {"ms_per_step": plain_ms, "value": world * args.systems / (plain_ms / 1000.0),
                       "speedup_of_headline": plain_ms / ms},
        "plain_fp64_per_node": (dict(per_node, speedup_of_headline=value / (world * per_node["value"]))
                                if per_node else None),
        "status_ok_fraction": ok,
        "fp64_resolve_fraction": float(np.mean((info & N.INFO_FP64_RESOLVE) != 0)),
        "mean_refine_passes_tensor_class": float(np.mean(((info >> N.INFO_REFINE_SHIFT) & 255)[p_all >= 33])),
        "fp64_factor": bool(args.fp64_factor) or bool(tuned and tuned.get("fp64_factor")),
        "autotune": tuned,
        "variants": variants,
        "plain_kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in plain_prof.items()},
        "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "legs": legs,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
