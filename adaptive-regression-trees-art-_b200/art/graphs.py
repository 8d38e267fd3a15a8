"""CUDA-graph replay of tree-level launch sequences.

A level's split search is one stream-ordered ``art_split_level`` sequence
(work-list planning, the persistent split kernel, per-node selection) with no
host synchronisation inside.  ``SplitLevelGraphs`` captures that sequence
once per shape class and replays it for every later level of the class:

* the class is (node capacity, row capacity, d_max, p_max, R, the splitter's
  scalar parameters, traces), capacities rounded up to powers of two;
* inputs are copied into the class's static device buffers, nodes beyond the
  level's K get zero rows (the kernel reports them as failed splits and they
  are never read back), and the static outputs are returned as views of the
  first K rows;
* every launch of the sequence reads the same buffers on every replay, so a
  replay computes exactly what the eager call computes on the same inputs.

The views are overwritten by the next replay of the same class: read a level
before splitting the next one (the builders do).  Capture runs with the
library's profiler off and with relaxed capture mode (the launchers query
occupancy and set kernel attributes, which are not stream work).
"""

from __future__ import annotations

import ctypes as C
from collections import OrderedDict

import numpy as np

from . import _native as N
from ._device import require_cuda, to_device, torch

__all__ = ["SplitLevelGraphs", "shared_split_graphs"]


def _pow2(v: int, floor: int) -> int:
    v = max(int(v), floor)
    return 1 << (v - 1).bit_length()


class _SplitGraph:
    def __init__(self, splitter, kcap, rcap, dmax, pmax, R, traces, kwargs):
        from .splitters import _level_result

        t = torch()
        dev = require_cuda()
        self.kcap, self.rcap, self.dmax, self.pmax, self.R = kcap, rcap, dmax, pmax, R
        lib = N.load_library()
        self.x = t.zeros(rcap * dmax, dtype=t.float64, device=dev)
        self.y = t.zeros(rcap, dtype=t.float64, device=dev)
        self.ro = t.zeros(kcap + 1, dtype=t.int64, device=dev)
        self.xo = t.zeros(kcap, dtype=t.int64, device=dev)
        self.dims = t.full((kcap,), dmax, dtype=t.int32, device=dev)
        self.feats = t.zeros(kcap, dtype=t.int32, device=dev)
        self.temp = t.ones(kcap, dtype=t.float64, device=dev)
        self.ridge = t.full((kcap,), 1e-6, dtype=t.float64, device=dev)
        self.parent = t.zeros(kcap, dtype=t.float64, device=dev)
        self.fallback = t.zeros(kcap, dtype=t.int8, device=dev)
        self.theta0 = t.zeros((kcap, R, dmax + 1), dtype=t.float64, device=dev)
        self.theta0[:, :, 0] = 1.0
        self.out = _level_result(kcap, R, int(splitter.max_iters), dmax, pmax, traces, dev)
        self.ws = t.empty(max(1, lib.art_split_workspace_size(kcap, R, dmax, pmax)), dtype=t.uint8, device=dev)
        self.splitter, self.traces, self.kwargs = splitter, traces, kwargs
        self.graph = None

    def _call(self, stream):
        from .splitters import split_level

        return split_level(self.splitter, self.x, self.y, self.ro, self.dims, self.feats, self.temp, self.ridge,
                           x_offsets=self.xo, parent_loss=self.parent, min_side_fallback=self.fallback,
                           theta0=self.theta0, traces=self.traces, max_dim=self.dmax, max_features=self.pmax,
                           out=self.out, workspace=self.ws, stream=stream, **self.kwargs)

    def capture(self):
        t = torch()
        was = N.profiling()
        if was:
            N.profile_enable(False)
        try:
            side = t.cuda.Stream()
            side.wait_stream(t.cuda.current_stream())
            with t.cuda.stream(side):
                self._call(side)  # warm-up outside capture: kernel attributes, lazy module load
            t.cuda.current_stream().wait_stream(side)
            t.cuda.synchronize()
            g = t.cuda.CUDAGraph()
            with t.cuda.graph(g, capture_error_mode="relaxed"):
                self._call(t.cuda.current_stream())
            self.graph = g
        finally:
            if was:
                N.profile_enable(True)

    def load(self, x, y, row_offsets, dims, feats, temp, ridge, parent, fallback, theta0):
        t = torch()
        K = int(dims.numel())
        rows = int(y.numel())
        self.x[: x.numel()].copy_(x, non_blocking=True)
        self.y[:rows].copy_(y, non_blocking=True)
        self.ro[: K + 1].copy_(row_offsets, non_blocking=True)
        self.ro[K + 1:].fill_(rows)
        nd = (row_offsets[1:] - row_offsets[:-1]) * dims.to(t.int64)  # rows of x per node, packed by node
        self.xo[:K].copy_(t.cumsum(nd, 0) - nd, non_blocking=True)
        self.xo[K:].fill_(rows * self.dmax)
        self.dims[:K].copy_(dims, non_blocking=True)
        self.dims[K:].fill_(self.dmax)
        self.feats[:K].copy_(feats, non_blocking=True)
        if K < self.kcap:
            self.feats[K:].copy_(feats[:1].expand(self.kcap - K), non_blocking=True)
        self.temp[:K].copy_(temp, non_blocking=True)
        self.ridge[:K].copy_(ridge, non_blocking=True)
        self.parent[:K].copy_(parent, non_blocking=True)
        self.fallback.zero_()
        self.fallback[:K].copy_(fallback, non_blocking=True)
        th = theta0.reshape(K, self.R, -1)
        self.theta0[:K, :, : th.shape[2]].copy_(th, non_blocking=True)
        if self.traces:  # the kernel writes only the iterations it ran
            self.out.trace_loss.fill_(float("nan"))
            self.out.trace_grad_norm.fill_(float("nan"))
            self.out.trace_step.fill_(float("nan"))
            self.out.trace_backtracks.fill_(-1)
        return K

    def view(self, K):
        from .splitters import LevelResult

        o = self.out
        res = LevelResult(*(getattr(o, f)[:K] for f in ("theta", "beta", "loss", "child_loss", "ridge_effective",
                                                      "n_right", "n_iters", "stop_reason", "failure", "flags",
                                                      "fallback_iteration", "final_alpha")))
        if self.traces:
            res.trace_loss, res.trace_step = o.trace_loss[:K], o.trace_step[:K]
            res.trace_backtracks, res.trace_grad_norm = o.trace_backtracks[:K], o.trace_grad_norm[:K]
        return res


class SplitLevelGraphs:
    """Per-shape-class captured split levels (least recently used dropped past ``capacity``)."""

    def __init__(self, capacity: int = 16):
        self.capacity = int(capacity)
        self._graphs: OrderedDict = OrderedDict()
        self.captures = 0
        self.replays = 0

    def split_level(self, splitter, x, y, row_offsets, dims, features, temperature, ridge, *, parent_loss,
                    min_side_fallback, theta0, hard_refit: bool = True, anneal_ratio: float = 1.0, seed: int = 0,
                    traces: bool = False, max_dim: int, max_features: int):
        """``splitters.split_level`` through a captured graph (same arguments, device or host arrays)."""

        from . import autotune
        from .splitters import split_params

        t = torch()
        dev = require_cuda()
        x = to_device(x, t.float64, dev).reshape(-1)
        y = to_device(y, t.float64, dev)
        ro = to_device(row_offsets, t.int64, dev)
        dims_t = to_device(dims, t.int32, dev)
        feats = to_device(features, t.int32, dev)
        K = int(dims_t.numel())
        R = int(max(1, splitter.n_restarts))
        temp = to_device(np.broadcast_to(np.asarray(temperature, float), (K,)).copy()
                         if not isinstance(temperature, t.Tensor) else temperature, t.float64, dev)
        rid = to_device(np.broadcast_to(np.asarray(ridge, float), (K,)).copy()
                        if not isinstance(ridge, t.Tensor) else ridge, t.float64, dev)
        pl = to_device(np.asarray(parent_loss, float).reshape(K) if not isinstance(parent_loss, t.Tensor)
                       else parent_loss, t.float64, dev)
        fb = to_device(np.broadcast_to(np.asarray(min_side_fallback, dtype=np.int8), (K,)).copy()
                       if not isinstance(min_side_fallback, t.Tensor) else min_side_fallback, t.int8, dev)
        th0 = to_device(theta0, t.float64, dev)
        if th0.reshape(K, R, -1).shape[2] > max_dim + 1:
            raise ValueError("theta0 rows are wider than max_dim + 1")
        kcap, rcap = _pow2(K, 8), _pow2(int(y.numel()), 4096)
        shape = autotune.cached_split_shape(int(max_dim), int(max_features), R)
        prm = split_params(splitter, hard_refit, anneal_ratio, seed, *shape)
        key = (kcap, rcap, int(max_dim), int(max_features), R, bytes(memoryview(prm)), bool(traces))
        g = self._graphs.get(key)
        if g is None:
            g = _SplitGraph(splitter, kcap, rcap, int(max_dim), int(max_features), R, bool(traces),
                            dict(hard_refit=hard_refit, anneal_ratio=anneal_ratio, seed=seed))
            g.load(x, y, ro, dims_t, feats, temp, rid, pl, fb, th0)
            g.capture()
            self.captures += 1
            self._graphs[key] = g
            while len(self._graphs) > self.capacity:
                self._graphs.popitem(last=False)
        else:
            self._graphs.move_to_end(key)
        g.load(x, y, ro, dims_t, feats, temp, rid, pl, fb, th0)
        g.graph.replay()
        self.replays += 1
        res = g.view(K)
        res._keepalive = (x, y, ro, dims_t, feats, temp, rid, pl, fb, th0)
        return res


_SHARED: dict[int, SplitLevelGraphs] = {}


def shared_split_graphs() -> SplitLevelGraphs:
    """The process-wide graph cache of the current device (reused across builds)."""

    dev = require_cuda()
    g = _SHARED.get(dev.index)
    if g is None:
        g = _SHARED[dev.index] = SplitLevelGraphs()
    return g
