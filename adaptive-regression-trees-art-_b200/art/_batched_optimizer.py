"""Resident batched split optimisation with fixed capacity (drop-in for the
reference ``art/_cuda_batched_optimizer.py:88-660``).

``BatchedOptimizerWorkspace`` keeps K equally sized node datasets (n rows, d
inputs) in device buffers and optimises any subset of them with one
``art_split_level`` launch sequence per call: every projected-gradient
iteration, line search, restart and the hard partition run on the device, and
the host reads the results once.  The reference drives the same loop from the
host with two device-to-host reads per iteration.

Initial states that are not supplied are drawn on the device (unit Gaussian w,
z = median(X w)), keyed by the workspace seed, a per-call counter and the
slot index, so the draws advance across calls as the reference's cuRAND
generator does and a slot's draws do not depend on the other slots selected.
"""

from __future__ import annotations

import numpy as np

from ._device import require_cuda, to_device, torch
from .models import AffineRidgeModel, PolynomialRidgeModel, kind_feature_count
from .optimizers import AdaptiveAlpha
from .splitters import (
    SplitNotFoundError,
    _model_kind,
    level_result_to_split,
    project_unit_w,
    split_level,
)


def _dimensions(*shape):
    """_cuda_batched_cholesky.py:15-19"""

    if any(not isinstance(v, (int, np.integer)) or not 0 < v <= np.iinfo(np.int32).max for v in shape):
        raise ValueError("Workspace dimensions must be positive CUDA integers.")
    return tuple(int(v) for v in shape)


def _node_ids(nodes, limit):
    """_cuda_batched_cholesky.py:22-28"""

    ids = np.asarray(nodes)
    if ids.ndim != 1 or (ids.size and not np.issubdtype(ids.dtype, np.integer)):
        raise ValueError("nodes must be a one-dimensional integer list.")
    if np.any(ids < 0) or np.any(ids >= limit) or len(np.unique(ids)) != len(ids):
        raise ValueError("nodes must contain distinct loaded slot indices.")
    return np.ascontiguousarray(ids, dtype=np.int64)


def _batch_data(X, y, temperature):
    """_cuda_batched_optimizer.py:45-56"""

    X, y = np.asarray(X, dtype=float), np.asarray(y, dtype=float)
    if X.ndim != 3 or min(X.shape) == 0 or y.shape != X.shape[:2]:
        raise ValueError("X/y must have nonempty shapes (K,n,d)/(K,n).")
    if not np.isfinite(X).all() or not np.isfinite(y).all():
        raise ValueError("X and y must be finite.")
    temperature = np.broadcast_to(np.asarray(temperature, dtype=float), (X.shape[0],))
    if not np.isfinite(temperature).all() or np.any(temperature <= 0):
        raise ValueError("Temperatures must be finite and positive.")
    _dimensions(*X.shape)
    return X, y, temperature


def _validate_settings(s, d, reorder):
    """_cuda_batched_optimizer.py:59-85"""

    if type(s.model_template) not in (AffineRidgeModel, PolynomialRidgeModel):
        raise TypeError("Batched Cholesky supports affine and polynomial ridge models.")
    if type(s.model_template) is PolynomialRidgeModel and (
            not isinstance(s.model_template.degree, (int, np.integer)) or s.model_template.degree not in (1, 2)):
        raise ValueError("Batched GPU features support only polynomial degree 1 or 2.")
    if s.refit_during_line_search:
        raise ValueError("Batched optimization requires refit_during_line_search=False and a resident optimizer.")
    if not isinstance(reorder, (bool, np.bool_)):
        raise ValueError("reorder must be a boolean.")
    s._validate_inputs(np.empty((0, d)), np.empty(0))
    for name in ("alpha0", "alpha_min", "alpha_max", "grad_atol", "grad_rtol", "weight_floor"):
        value = getattr(s, name)
        if not np.isfinite(value) or value < 0 or (name.startswith("alpha") and value == 0):
            raise ValueError(f"Invalid {name}.")
    for name, minimum in (("max_iters", 0), ("max_backtracks", 0), ("Xw_refresh", 0),
                          ("backtrack_batch_size", 1), ("max_line_search_failures", 1), ("n_restarts", 0)):
        if not isinstance(getattr(s, name), (int, np.integer)) or getattr(s, name) < minimum:
            raise ValueError(f"Invalid {name}.")
    if not 0 < s.rho < 1 or not 0 < s.armijo_c < 1:
        raise ValueError("rho and armijo_c must lie strictly between 0 and 1.")
    if not np.isfinite(s.model_template.ridge) or s.model_template.ridge < 0:
        raise ValueError("ridge must be finite and nonnegative.")
    AdaptiveAlpha(s.alpha0, s.alpha_min, s.alpha_max, s.alpha_grow, s.alpha_recovery, s.heavy_backtrack_threshold)


class BatchedOptimizerWorkspace:
    """Allocate capacity K once; load and optimize cohorts of k <= K nodes.

    X/y are NumPy (k,n,d)/(k,n); temperatures may vary by node.  optimize()
    returns a list in requested slot order (all k by default), each entry a
    SplitResult or SplitNotFoundError, holding CPU data only.  Settings and
    n/d stay fixed; use load() to replace data.  A workspace is used serially
    on the device (and stream) it was created on.  ``reorder`` is accepted for
    the reference's signature; the device work list already skips finished
    restarts, so it does not change results.
    """

    def __init__(self, splitter, X, y, *, temperature=None, reorder=True):
        temp = splitter.temperature if temperature is None else temperature
        X, y, temp = _batch_data(X, y, temp)
        self._allocate(splitter, *X.shape, reorder=reorder)
        self._load(X, y, temp)

    @classmethod
    def allocate(cls, splitter, capacity, n, d, *, reorder=True, stream=None):
        """Reserve device and host buffers for an entire build."""

        ws = cls.__new__(cls)
        ws._allocate(splitter, capacity, n, d, reorder=reorder, stream=stream)
        return ws

    def _allocate(self, splitter, capacity, n, d, *, reorder, stream=None):
        self.K, self.n, self.d = _dimensions(capacity, n, d)
        _validate_settings(splitter, self.d, reorder)
        self.s, self.capacity, self.k = splitter, self.K, 0
        self.reorder = bool(reorder)
        self.seed = int(splitter._rng().integers(0, np.iinfo(np.int64).max))
        self.required = splitter._required_side_points(self.n)
        self.stream = stream
        self._calls = 0
        self._host_rng = np.random.default_rng(self.seed)
        t = torch()
        self.device = require_cuda()
        self.x = t.empty((self.K, self.n, self.d), dtype=t.float64, device=self.device)
        self.y_dev = t.empty((self.K, self.n), dtype=t.float64, device=self.device)
        self.host_X = np.empty((self.K, self.n, self.d))
        self.host_y = np.empty((self.K, self.n))
        self.temperature = np.ones(self.K)
        self.X, self.y = self.host_X[:0], self.host_y[:0]
        self.kind = _model_kind(splitter.model_template)
        self.p = kind_feature_count(self.d, self.kind)
        self._open = True

    def _check_open(self):
        if not getattr(self, "_open", False):
            raise RuntimeError("The workspace is closed.")
        t = torch()
        if t.cuda.current_device() != self.device.index:
            raise ValueError("Use the workspace on the device where it was created.")

    def load(self, X, y, *, temperature=None):
        """Load one packed CPU cohort into the fixed device buffers.

        Shapes are (k,n,d)/(k,n), 0<k<=capacity.  Builders may pack directly
        into host_X/host_y and pass their occupied prefixes."""

        self._check_open()
        temp = self.s.temperature if temperature is None else temperature
        X, y, temp = _batch_data(X, y, temp)
        if X.shape[0] > self.K or X.shape[1:] != (self.n, self.d):
            raise ValueError("X/y must have shapes (k,n,d)/(k,n), 0<k<=capacity.")
        return self._load(X, y, temp)

    def _load(self, X, y, temp):
        k = X.shape[0]
        for dst, src in ((self.host_X[:k], X), (self.host_y[:k], y)):
            if dst.ctypes.data != src.ctypes.data or dst.strides != src.strides:
                np.copyto(dst, src)
        self.temperature[:k] = temp
        self.x[:k].copy_(to_device(self.host_X[:k], torch().float64, self.device))
        self.y_dev[:k].copy_(to_device(self.host_y[:k], torch().float64, self.device))
        self.k = k
        self.X, self.y = self.host_X[:k], self.host_y[:k]
        return self

    def _random_start(self, j):
        """Unit Gaussian w and z = median(X w) of slot j (splitters.py:692-700)."""

        w = self._host_rng.normal(size=self.d)
        nrm = np.linalg.norm(w)
        if nrm <= 1e-12:
            w[:] = 0.0
            w[0], nrm = 1.0, 1.0
        w = w / nrm
        return np.concatenate([w, [float(np.median(self.host_X[j] @ w))]])

    def _parent_losses(self, ids):
        """Mean squared residual of each selected node's unweighted ridge fit and
        whether that fit succeeded (the reference's _parent_loss, :609-626)."""

        from .models import segment_residuals, solve_weighted_ridge_batched

        t = torch()
        count = len(ids)
        sel = t.as_tensor(ids, device=self.device)
        ro = np.arange(count + 1, dtype=np.int64) * self.n
        x = self.x.index_select(0, sel).reshape(-1)
        y = self.y_dev.index_select(0, sel).reshape(-1)
        out = solve_weighted_ridge_batched(x, y, None, ro, [self.d] * count, [self.kind] * count,
                                           float(self.s.model_template.ridge), weight_floor=0.0,
                                           solver="normal", precision="fp64", max_features=self.p,
                                           max_dim=self.d, stream=self.stream)
        beta = t.nan_to_num(out.beta, nan=0.0)
        sse, _ = segment_residuals(x, y, ro, [self.d] * count, [self.kind] * count, beta, stream=self.stream)
        ok = (out.status == 0).cpu().numpy()
        return (sse / self.n).cpu().numpy(), ok

    def optimize(self, theta0=None, *, parent_loss=None, nodes=None, min_side_fallback=None, hard_refit=True):
        """Run restarts on the device and export the best split of each node once.

        nodes selects occupied slot IDs, in return order; default is all k.
        For r selected nodes, theta0 is (r,d+1) or (R,r,d+1) (a 2-D theta0
        starts restart 0 only; the others draw their own starts), and
        parent_loss is (r,).  min_side_fallback overrides the splitter's
        policy for this call.  hard_refit=False (one restart only) returns
        geometry and counts without hard models or loss measurements."""

        self._check_open()
        if not self.k:
            raise RuntimeError("Load data before optimizing.")
        ids = np.arange(self.k, dtype=np.int64) if nodes is None else _node_ids(nodes, self.k)
        count = len(ids)
        R = max(1, int(self.s.n_restarts))
        if not isinstance(hard_refit, (bool, np.bool_)):
            raise ValueError("hard_refit must be a boolean.")
        if not hard_refit and self.s.n_restarts != 1:
            raise ValueError("Skipping hard refits requires n_restarts == 1.")
        initial = None if theta0 is None else np.asarray(theta0, dtype=float)
        if initial is not None and (initial.shape not in ((count, self.d + 1), (R, count, self.d + 1))
                                    or not np.isfinite(initial).all()):
            raise ValueError("theta0 must be finite with shape (r,d+1) or (R,r,d+1).")
        if parent_loss is not None:
            parent_loss = np.asarray(parent_loss, dtype=float)
            if parent_loss.shape != (count,) or not np.isfinite(parent_loss).all() or np.any(parent_loss < 0):
                raise ValueError("parent_loss must be finite and nonnegative with shape (r,).")
        if min_side_fallback is not None and not isinstance(min_side_fallback, (bool, np.bool_)):
            raise ValueError("min_side_fallback must be a boolean.")
        if not count:
            return []
        if parent_loss is None:
            parent_loss, parent_ok = self._parent_losses(ids)
        else:
            parent_ok = np.ones(count, bool)
        th0 = None
        if initial is not None:
            th0 = np.empty((count, R, self.d + 1))
            for r in range(R):
                for c, j in enumerate(ids):
                    if initial.ndim == 3:
                        th0[c, r] = project_unit_w(initial[r, c])
                    elif r == 0:
                        th0[c, r] = project_unit_w(initial[c])
                    else:
                        th0[c, r] = self._random_start(int(j))
        t = torch()
        sel = t.as_tensor(ids, device=self.device)
        fallback = self.s.min_side_fallback if min_side_fallback is None else bool(min_side_fallback)
        self._calls += 1
        res = split_level(self.s, self.x.index_select(0, sel).reshape(-1), self.y_dev.index_select(0, sel).reshape(-1),
                          np.arange(count + 1, dtype=np.int64) * self.n, [self.d] * count, [self.kind] * count,
                          self.temperature[ids], float(self.s.model_template.ridge), parent_loss=parent_loss,
                          min_side_fallback=[int(fallback)] * count, theta0=th0, hard_refit=bool(hard_refit),
                          seed=(self.seed + self._calls) & ((1 << 63) - 1), traces=True,
                          node_keys=ids.astype(np.uint64), max_dim=self.d, max_features=self.p,
                          stream=self.stream)
        out = []
        for c in range(count):
            if not parent_ok[c]:
                out.append(SplitNotFoundError("cholesky_failure", "Parent Cholesky fit failed."))
                continue
            try:
                r = level_result_to_split(self.s, res, c, self.n, float(parent_loss[c]), bool(hard_refit))
                r.metadata.update(optimizer="b200_batched", temperature=float(self.temperature[ids[c]]),
                                  initialization="gpu" if initial is None else "provided")
                out.append(r)
            except SplitNotFoundError as exc:
                out.append(exc)
        return out

    def close(self):
        if getattr(self, "_open", False):
            self._open = False
            self.x = self.y_dev = None
            self.host_X = self.host_y = None
            self.X = self.y = None
            self.k = 0

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optimize_batch(splitter, X, y, *, theta0=None, parent_loss=None, temperature=None, reorder=True,
                   hard_refit=True):
    """Convenience entry point (_cuda_batched_optimizer.py:655-660); use the
    workspace directly to reuse its buffers."""

    with BatchedOptimizerWorkspace(splitter, X, y, temperature=temperature, reorder=reorder) as ws:
        return ws.optimize(theta0, parent_loss=parent_loss, hard_refit=hard_refit)
