"""Device-measured choice of the batched kernels' launch shapes.

Two choices are tuned by timing the library itself on a sample of the
caller's own batch, with CUDA events on the launching stream:

* ``ridge_tensor_min_features`` -- in the mixed ridge form, the smallest
  feature count p solved by the tensor-core kernel; smaller systems take the
  FP64 kernels.  Each feature class p >= 33 of the sample is timed on the
  FP64 kernels and on the tensor-core kernel with its FP32 and its FP64
  factorisation; the threshold is the smallest p from which the tensor-core
  kernel wins for every larger class, and the factorisation is the one with
  the lower total time over the tensor classes.
* ``split_shape`` for a (d, p, R) split level -- either the CTA form, with
  the restarts that share one CTA's row passes (``group_restarts``), the
  Armijo step sizes evaluated per trial pass (``trial_steps``) and the
  resident CTAs per SM (``ctas_per_sm``: one with the deepest row ring, or
  two with half the shared memory and a 128-register cap), or the
  warp-per-restart form (``restart_warps``) with its trial steps; each
  candidate runs the sample level and the fastest is kept.

Results live in an in-process table keyed by the device (name, SM count,
compute capability), persisted as JSON at ``$ART_AUTOTUNE_CACHE`` when that
is set.  Lookups (``cached_*``) read only host-known keys, never device
data, so they add no synchronisation to a call; an untuned key returns the
library default.  Tuning itself synchronises and is meant for warm-up.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import numpy as np

from ._device import require_cuda, to_device, torch

__all__ = ["device_key", "cached_ridge_threshold", "cached_split_shape", "tune_ridge_threshold",
           "tune_split_shape", "clear", "table"]

_TABLE: dict[str, dict] = {}
_LOCK = threading.Lock()
_LOADED = False
NO_TENSOR = 161  # threshold above every tensor-core feature count


def device_key() -> str:
    t = torch()
    dev = require_cuda()
    props = t.cuda.get_device_properties(dev)
    return f"{props.name}|sm{props.multi_processor_count}|cc{props.major}.{props.minor}"


def _cache_path() -> Path | None:
    p = os.environ.get("ART_AUTOTUNE_CACHE")
    return Path(p) if p else None


def _load() -> None:
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    path = _cache_path()
    if path is not None and path.exists():
        try:
            _TABLE.update(json.loads(path.read_text()))
        except (OSError, ValueError):
            pass


def _store(key: str, value: dict) -> None:
    with _LOCK:
        _TABLE[key] = value
        path = _cache_path()
        if path is not None:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_suffix(".tmp")
            tmp.write_text(json.dumps(_TABLE, indent=1, sort_keys=True))
            os.replace(tmp, path)


def clear() -> None:
    with _LOCK:
        _TABLE.clear()


def table() -> dict:
    _load()
    return dict(_TABLE)


def _ridge_key() -> str:
    return f"ridge|{device_key()}"


def _split_key(d: int, p: int, R: int) -> str:
    return f"split|{device_key()}|d={int(d)}|p={int(p)}|R={int(R)}"


def cached_ridge_choice() -> tuple[int, bool | None]:
    """Tuned (tensor-core threshold, FP64 factorisation) for this device, or (0, None)."""

    _load()
    try:
        entry = _TABLE.get(_ridge_key())
    except RuntimeError:
        return 0, None
    if not entry:
        return 0, None
    return int(entry["tensor_min_features"]), bool(entry.get("fp64_factor", False))


def cached_ridge_threshold(dims=None, features=None, row_offsets=None, fp64_factor: bool = False) -> int:
    """Tuned tensor-core threshold for this device, or 0 (library default)."""

    return cached_ridge_choice()[0]


def cached_split_shape(d: int, p: int, R: int) -> tuple[int, int, int, int]:
    """Tuned (group_restarts, trial_steps, ctas_per_sm, restart_warps) for a
    (d, p, R) level; untuned: (0, 0, 0, 1), the warp-per-restart form (the
    library takes the CTA form where the level does not fit it)."""

    _load()
    try:
        entry = _TABLE.get(_split_key(d, p, R))
    except RuntimeError:
        return 0, 0, 0, 1
    if not entry:
        return 0, 0, 0, 1
    return (int(entry["group_restarts"]), int(entry["trial_steps"]), int(entry.get("ctas_per_sm", 0)),
            int(entry.get("restart_warps", 0)))


def _event_time(fn, repeats: int, stream) -> float:
    t = torch()
    fn()
    t.cuda.synchronize()
    best = float("inf")
    for _ in range(repeats):
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        t.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _subset(x, y, w, row_offsets, x_offsets, dims, kinds, ridge, idx):
    """Gather systems ``idx`` into a contiguous batch (device tensors)."""

    t = torch()
    dev = x.device
    ro = row_offsets.cpu().numpy() if isinstance(row_offsets, t.Tensor) else np.asarray(row_offsets)
    xo = x_offsets.cpu().numpy() if isinstance(x_offsets, t.Tensor) else np.asarray(x_offsets)
    dh = dims.cpu().numpy() if isinstance(dims, t.Tensor) else np.asarray(dims)
    n = ro[idx + 1] - ro[idx]
    rows = np.concatenate([np.arange(ro[k], ro[k + 1]) for k in idx]) if len(idx) else np.zeros(0, np.int64)
    xel = np.concatenate([np.arange(xo[k], xo[k] + (ro[k + 1] - ro[k]) * dh[k]) for k in idx]) \
        if len(idx) else np.zeros(0, np.int64)
    rows_t = t.from_numpy(rows).to(dev)
    xel_t = t.from_numpy(xel).to(dev)
    new_ro = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    new_xo = np.concatenate([[0], np.cumsum(n * dh[idx])])[:-1].astype(np.int64)
    sub = dict(x=x[xel_t], y=y[rows_t], w=None if w is None else w[rows_t],
               row_offsets=t.from_numpy(new_ro).to(dev), x_offsets=t.from_numpy(new_xo).to(dev),
               dims=t.from_numpy(np.ascontiguousarray(dh[idx]).astype(np.int32)).to(dev))
    kd = kinds.cpu().numpy() if isinstance(kinds, t.Tensor) else np.asarray(kinds)
    sub["kinds"] = t.from_numpy(np.ascontiguousarray(kd[idx]).astype(np.int32)).to(dev)
    rh = ridge.cpu().numpy() if isinstance(ridge, t.Tensor) else np.broadcast_to(np.asarray(ridge, float), dh.shape)
    sub["ridge"] = t.from_numpy(np.ascontiguousarray(rh[idx]).astype(np.float64)).to(dev)
    return sub


def tune_ridge_threshold(x, y, w, row_offsets, dims, kinds, ridge, *, x_offsets=None, max_dim=None,
                         fp64_factor: bool | None = None, per_class: int = 512, repeats: int = 3, seed: int = 0,
                         stream=None) -> dict:
    """Time each tensor-eligible feature class on every route; store and return the choice.
    ``fp64_factor`` None tunes the factorisation too, a bool fixes it."""

    from .models import kind_feature_count, solve_weighted_ridge_batched

    t = torch()
    dev = require_cuda()
    stream = t.cuda.current_stream() if stream is None else stream
    x = to_device(x, t.float64, dev)
    y = to_device(y, t.float64, dev)
    w = None if w is None else to_device(w, t.float64, dev)
    dh = dims.cpu().numpy() if isinstance(dims, t.Tensor) else np.asarray(dims)
    kh = kinds.cpu().numpy() if isinstance(kinds, t.Tensor) else np.asarray(kinds)
    if x_offsets is None:
        ro = row_offsets.cpu().numpy() if isinstance(row_offsets, t.Tensor) else np.asarray(row_offsets)
        x_offsets = ro[:-1] * dh
    p_all = np.array([kind_feature_count(int(a), int(b)) for a, b in zip(dh, kh)])
    rng = np.random.default_rng(seed)
    timings = {}
    for p in sorted(set(int(v) for v in p_all if 33 <= v <= 160)):
        members = np.flatnonzero(p_all == p)
        idx = np.sort(rng.choice(members, size=min(per_class, members.size), replace=False))
        sub = _subset(x, y, w, row_offsets, x_offsets, dims, kinds, ridge, idx)
        md = int(max_dim) if max_dim is not None else int(dh.max())

        def run(threshold, factor, sub=sub, p=p, md=md):
            return solve_weighted_ridge_batched(
                sub["x"], sub["y"], sub["w"], sub["row_offsets"], sub["dims"], sub["kinds"], sub["ridge"],
                x_offsets=sub["x_offsets"], precision="mixed", max_features=p, max_dim=md,
                fp64_factor=factor, tensor_min_features=threshold, stream=stream)

        tm = {"fp64_ms": _event_time(lambda: run(NO_TENSOR, False), repeats, stream), "systems": int(idx.size)}
        for factor in ((False, True) if fp64_factor is None else (bool(fp64_factor),)):
            key = "tensor_f64factor_ms" if factor else "tensor_ms"
            tm[key] = _event_time(lambda: run(p, factor), repeats, stream)
        timings[p] = tm
    # factorisation: lower total tensor-core time over the classes
    if fp64_factor is None:
        f32 = sum(v["tensor_ms"] for v in timings.values())
        f64 = sum(v["tensor_f64factor_ms"] for v in timings.values())
        factor = bool(f64 < f32)
    else:
        factor = bool(fp64_factor)
    tkey = "tensor_f64factor_ms" if factor else "tensor_ms"
    choice = NO_TENSOR
    for p in sorted(timings, reverse=True):
        if timings[p][tkey] < timings[p]["fp64_ms"]:
            choice = p
        else:
            break
    entry = {"tensor_min_features": int(choice), "fp64_factor": factor,
             "classes": {str(k): v for k, v in timings.items()}}
    _store(_ridge_key(), entry)
    return entry


WARP_MAX_DIM = 23       # warp-per-restart form: inputs, features and trial steps it takes
WARP_MAX_FEATURES = 23
WARP_MAX_TRIALS = 8


def split_candidates(R: int, max_backtracks: int, d: int = 0, p: int = 0,
                     tensor_gram: bool = False) -> list[tuple[int, int, int, int]]:
    """(group_restarts, trial_steps, ctas_per_sm, restart_warps) shapes tried
    for R restarts.

    Two CTAs per SM are tried for groups of at most 8 restarts: a group of 16
    keeps 16 restarts' state per thread, which the 128-register cap spills.
    The warp-per-restart form is tried when the level fits it (d and p at
    most 23, no tensor-core Gram)."""

    groups = sorted({g for g in (R, 16, 8, 4, 2, 1) if 1 <= g <= min(R, 16)}, reverse=True)
    out = []
    for g in groups:
        hmax = min(32, max(1, 256 // g), max_backtracks + 1)
        for h in sorted({min(hmax, v) for v in (2, 4, 8, 16)}, reverse=True):
            for c in ((1, 2) if g <= 8 else (1,)):
                out.append((g, h, c, 0))
    if not tensor_gram and 1 <= d <= WARP_MAX_DIM and 1 <= p <= WARP_MAX_FEATURES:
        hmax = min(WARP_MAX_TRIALS, max_backtracks + 1)
        for h in sorted({min(hmax, v) for v in (1, 2, 4)}, reverse=True):
            out.append((0, h, 0, 1))
    return out


def tune_split_shape(splitter, x, y, row_offsets, dims, features, temperature, ridge, *, max_dim: int,
                     max_features: int, theta0=None, anneal_ratio: float = 1.0, hard_refit: bool = True,
                     repeats: int = 2, stream=None) -> dict:
    """Time the candidate launch shapes on this level; store and return the fastest."""

    from .splitters import split_level

    t = torch()
    stream = t.cuda.current_stream() if stream is None else stream
    R = int(max(1, splitter.n_restarts))
    tc = bool(getattr(splitter, "tensor_gram", False)) and getattr(splitter, "precision", "fp64") == "mixed"
    timings = {}
    for g, h, c, w in split_candidates(R, int(splitter.max_backtracks), int(max_dim), int(max_features), tc):
        def run(g=g, h=h, c=c, w=w):
            return split_level(splitter, x, y, row_offsets, dims, features, temperature, ridge, theta0=theta0,
                               anneal_ratio=anneal_ratio, hard_refit=hard_refit, max_dim=max_dim,
                               max_features=max_features, group_restarts=g, trial_steps=h, ctas_per_sm=c,
                               restart_warps=w, stream=stream)

        timings[f"{g}x{h}x{c}x{w}"] = _event_time(run, repeats, stream)
    best = min(timings, key=timings.get)
    g, h, c, w = (int(v) for v in best.split("x"))
    entry = {"group_restarts": g, "trial_steps": h, "ctas_per_sm": c, "restart_warps": w,
             "candidates_ms": timings}
    _store(_split_key(max_dim, max_features, R), entry)
    return entry
