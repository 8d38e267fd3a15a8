"""Soft oblique split search on the GPU (drop-in for the reference art/splitters.py).

``SoftObliqueSplitter.split`` (splitters.py:252-363) runs the whole projected
gradient loop for one node in ``art_split_level``; ``split_level`` runs a
whole tree level (many nodes, uneven sizes) in one launch sequence and is
what the BFS builder dispatches.  Child models of the soft objective are
normal-equation Cholesky fits (a failed factorisation marks the restart as
``cholesky_failure``, as the reference's batched GPU form does).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Literal, Protocol, runtime_checkable

import numpy as np

from . import _native as N
from ._device import WORKSPACES, ptr, require_cuda, stream_handle, to_device, torch
from .metrics import mean_squared_error
from .models import (
    AffineRidgeModel,
    PolynomialRidgeModel,
    PreparedDesign,
    RegressionModel,
    RidgeSolveResult,
    WeightedRegressionModel,
    kind_feature_count,
)
from .timing import BuildTimingProfile, SplitterTimingProfile

# largest total size of the row copies one split_temperatures launch holds
TEMPERATURE_BATCH_BYTES = 256 << 20

Optimizer = Literal["b200", "cpu", "hybrid_gram", "cupy_qr", "cupy_cholesky", "cupy_batched_cholesky"]
OPTIMIZERS = ("b200", "cpu", "hybrid_gram", "cupy_qr", "cupy_cholesky", "cupy_batched_cholesky")


class SplitNotFoundError(RuntimeError):
    """Raised when all splitter attempts produce an invalid hard partition (splitters.py:36-53)."""

    def __init__(self, reason: str, message: str, diagnostics: dict[str, Any] | None = None,
                 restarts_on_failure: int = 0, failure_reasons: tuple[str, ...] = (),
                 context: dict[str, Any] | None = None):
        super().__init__(message)
        self.reason = reason
        self.diagnostics = diagnostics
        self.restarts_on_failure = int(restarts_on_failure)
        self.failure_reasons = tuple(failure_reasons)
        self.context = {} if context is None else dict(context)


@runtime_checkable
class Splitter(Protocol):
    def split(self, X: np.ndarray, y: np.ndarray, parent_model: RegressionModel | None = None,
              parent_loss: float | None = None, prepared_design: PreparedDesign | None = None) -> "SplitResult": ...


def project_unit_w(theta: np.ndarray) -> np.ndarray:
    """Project theta = [w, z] onto ||w|| = 1 (splitters.py:71-83)."""

    theta = np.asarray(theta, dtype=float).reshape(-1)
    if theta.size < 2:
        raise ValueError("theta must contain at least one w component and one z component.")
    n = np.linalg.norm(theta[:-1])
    if n <= 1e-12:
        raise ValueError("Cannot project theta with near-zero w.")
    out = theta.copy()
    out[:-1] = theta[:-1] / n
    return out


def project_unit_w_gradient(theta: np.ndarray, grad: np.ndarray) -> np.ndarray:
    """Tangent-space projection of the w-gradient (splitters.py:86-98)."""

    theta = project_unit_w(theta)
    grad = np.asarray(grad, dtype=float).reshape(-1)
    if grad.shape != theta.shape:
        raise ValueError("grad and theta must have the same shape.")
    w = theta[:-1]
    out = grad.copy()
    out[:-1] = grad[:-1] - float(grad[:-1] @ w) * w
    return out


@dataclass
class SplitResult:
    """A split, optionally carrying hard models and their measured loss (splitters.py:114-196)."""

    w: np.ndarray
    z: float
    left_model: RegressionModel | None
    right_model: RegressionModel | None
    loss: float | None
    parent_loss: float
    split_gain: float | None
    relative_split_gain: float | None
    n_left: int
    n_right: int
    converged: bool
    n_iters: int
    stop_reason: str
    metadata: dict[str, Any] = field(default_factory=dict)

    @property
    def has_hard_fit(self) -> bool:
        return self.loss is not None

    def predict(self, X: np.ndarray) -> np.ndarray:
        if not self.has_hard_fit:
            raise RuntimeError("This partition has no hard models; top up and fit its children first.")
        X = np.asarray(X, dtype=float)
        if X.ndim == 1:
            X = X.reshape(1, -1)
        right = (X @ self.w - self.z) >= 0.0
        out = np.empty(X.shape[0])
        if np.any(~right):
            out[~right] = self.left_model.predict(X[~right])
        if np.any(right):
            out[right] = self.right_model.predict(X[right])
        return out


def _model_kind(model) -> int:
    if type(model) is AffineRidgeModel:
        return N.FEATURES_AFFINE
    if type(model) is PolynomialRidgeModel and model.degree in (1, 2):
        return model.kind()
    raise TypeError("the GPU split search supports AffineRidgeModel and degree 1/2 PolynomialRidgeModel")


def _clone_with(model, coef, lam):
    m = model.clone()
    m.coef_ = np.asarray(coef, dtype=float).copy()
    m.solve_result_ = RidgeSolveResult(coefficients=m.coef_, solver_requested=getattr(model, "solver", "normal"),
                                       solver_used="cholesky", condition_estimator=None, cond_estimate=None,
                                       ridge_effective=float(lam))
    return m


@dataclass
class LevelResult:
    """Device outputs of one ``split_level`` call (torch tensors)."""

    theta: object
    beta: object
    loss: object
    child_loss: object
    ridge_effective: object
    n_right: object
    n_iters: object
    stop_reason: object
    failure: object
    flags: object
    fallback_iteration: object
    final_alpha: object
    trace_loss: object | None = None
    trace_step: object | None = None
    trace_backtracks: object | None = None
    trace_grad_norm: object | None = None


def split_params(s: "SoftObliqueSplitter", hard_refit: bool, anneal_ratio: float = 1.0, seed: int = 0,
                 group_restarts: int = 0, trial_steps: int = 0, ctas_per_sm: int = 0, restart_warps: int = 0):
    """ArtSplitParams of a splitter.  ``precision="mixed"`` evaluates the
    sigmoid gates in single precision (objective within 1e-5 relative of the
    FP64 form); solves and the side decisions stay FP64, and the soft-pass
    side Grams are FP64 sums, or tensor-core TF32 hi/lo products with
    ``tensor_gram=True``."""

    if getattr(s, "precision", "fp64") not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'.")
    return N.ArtSplitParams(
        int(s.max_iters), int(max(1, s.n_restarts)), float(s.grad_atol), float(s.grad_rtol),
        int(s.min_side_points), float(s.min_side_fraction), float(s.alpha0), float(s.rho),
        float(s.armijo_c), int(s.max_backtracks), int(bool(s.adaptive_alpha)), float(s.alpha_min),
        float(s.alpha_max), float(s.alpha_grow), float(s.alpha_recovery), int(s.heavy_backtrack_threshold),
        int(s.max_line_search_failures), float(s.weight_floor), int(bool(hard_refit)),
        N.PRECISION_MIXED if getattr(s, "precision", "fp64") == "mixed" else N.PRECISION_FP64,
        float(anneal_ratio), int(seed) & ((1 << 64) - 1), int(group_restarts), int(trial_steps),
        int(ctas_per_sm), int(bool(getattr(s, "tensor_gram", False)) and getattr(s, "precision", "fp64") == "mixed"),
        int(bool(restart_warps)))


def split_level(splitter: "SoftObliqueSplitter", x, y, row_offsets, dims, features, temperature, ridge,
                *, x_offsets=None, parent_loss=None, min_side_fallback=None, theta0=None,
                hard_refit: bool = True, anneal_ratio: float = 1.0, seed: int = 0, traces: bool = False,
                max_dim: int | None = None, max_features: int | None = None, node_keys=None,
                group_restarts: int | None = None, trial_steps: int | None = None,
                ctas_per_sm: int | None = None, restart_warps: int | None = None, min_side_points=None,
                out: LevelResult | None = None, workspace=None, stream=None) -> LevelResult:
    """Split K nodes in one launch sequence; arrays are numpy or torch (moved to the device).

    theta0, when given, is (K, R, d_max + 1); otherwise restarts start from
    device draws keyed by ``seed`` and the node's position k (unit Gaussian w,
    z = median(X w)), or by ``node_keys[k]`` (uint64 per node) when given, so
    that a node's draws do not depend on the batch it is solved in.
    ``group_restarts`` / ``trial_steps`` / ``ctas_per_sm`` / ``restart_warps``
    fix the kernel's launch shape (restarts per CTA, Armijo steps per trial
    pass, resident CTAs per SM, or one warp per restart); None takes the
    autotuned choice for (d, p, R) on this device, else the library's.
    ``min_side_points`` (K ints) overrides the splitter's minimum side count
    per node, so nodes with different limits share one launch.
    ``out`` (a LevelResult of K rows) and ``workspace`` (a uint8 device
    tensor of at least ``art_split_workspace_size`` bytes) make the call
    allocate nothing, as a captured graph needs.
    """

    t = torch()
    lib = N.load_library()
    dev = require_cuda()
    x = to_device(x, t.float64, dev)
    y = to_device(y, t.float64, dev)
    ro = to_device(row_offsets, t.int64, dev)
    dims_t = to_device(dims, t.int32, dev)
    feats = to_device(features, t.int32, dev)
    K = int(dims_t.numel())
    R = int(max(1, splitter.n_restarts))
    if x_offsets is None:
        x_offsets = ro[:-1] * dims_t.to(t.int64)
    xo = to_device(x_offsets, t.int64, dev)
    temp = to_device(np.broadcast_to(np.asarray(temperature, float), (K,)).copy() if not isinstance(temperature, t.Tensor) else temperature, t.float64, dev)
    rid = to_device(np.broadcast_to(np.asarray(ridge, float), (K,)).copy() if not isinstance(ridge, t.Tensor) else ridge, t.float64, dev)
    pl = None if parent_loss is None else to_device(np.asarray(parent_loss, float).reshape(K) if not isinstance(parent_loss, t.Tensor) else parent_loss, t.float64, dev)
    fb = None
    if isinstance(min_side_fallback, t.Tensor):
        fb = to_device(min_side_fallback, t.int8, dev)
    elif min_side_fallback is not None:
        fb = to_device(np.broadcast_to(np.asarray(min_side_fallback, dtype=np.int8), (K,)).copy(), t.int8, dev)
    elif splitter.min_side_fallback:
        fb = t.ones(K, dtype=t.int8, device=dev)
    if max_dim is None or max_features is None:
        dh, fh = dims_t.cpu().numpy(), feats.cpu().numpy()
        max_dim = int(dh.max()) if max_dim is None else max_dim
        max_features = max(kind_feature_count(int(a), int(b)) for a, b in zip(dh, fh)) if max_features is None else max_features
    th0 = None
    stride = max_dim + 1
    if theta0 is not None:
        th0 = to_device(theta0, t.float64, dev).reshape(K * R, -1).contiguous()
        stride = int(th0.shape[1])
    M = int(splitter.max_iters)
    if out is None:
        out = _level_result(K, R, M, int(max_dim), int(max_features), traces, dev)
    nk = None
    if node_keys is not None:
        nk = to_device(np.asarray(node_keys, dtype=np.uint64).view(np.int64) if not isinstance(node_keys, t.Tensor)
                       else node_keys, t.int64, dev)
    seg = N.ArtSegments(K, ptr(ro), ptr(xo), ptr(dims_t), ptr(feats))
    ms = None
    if min_side_points is not None:
        ms = to_device(np.asarray(min_side_points, dtype=np.int32).reshape(K) if not isinstance(min_side_points, t.Tensor)
                       else min_side_points, t.int32, dev)
    prob = N.ArtSplitProblem(seg, ptr(x), ptr(y), ptr(temp), ptr(rid), ptr(pl), ptr(fb), ptr(th0), stride,
                             int(max_dim), int(max_features), ptr(nk), ptr(ms))
    if group_restarts is None or trial_steps is None or ctas_per_sm is None or restart_warps is None:
        from . import autotune

        g_auto, h_auto, c_auto, w_auto = autotune.cached_split_shape(int(max_dim), int(max_features), R)
        group_restarts = g_auto if group_restarts is None else group_restarts
        trial_steps = h_auto if trial_steps is None else trial_steps
        ctas_per_sm = c_auto if ctas_per_sm is None else ctas_per_sm
        restart_warps = w_auto if restart_warps is None else restart_warps
    prm = split_params(splitter, hard_refit, anneal_ratio, seed, group_restarts, trial_steps, ctas_per_sm,
                       restart_warps)
    res = N.ArtSplitResult(ptr(out.theta), int(out.theta.shape[1]), ptr(out.beta), int(out.beta.shape[2]),
                           ptr(out.loss), ptr(out.child_loss), ptr(out.ridge_effective), ptr(out.n_right),
                           ptr(out.n_iters), ptr(out.stop_reason), ptr(out.failure), ptr(out.flags),
                           ptr(out.fallback_iteration), ptr(out.final_alpha), ptr(out.trace_loss),
                           ptr(out.trace_step), ptr(out.trace_backtracks), ptr(out.trace_grad_norm))
    nbytes = lib.art_split_workspace_size(K, R, int(max_dim), int(max_features))
    ws = WORKSPACES.get(nbytes, stream) if workspace is None else workspace
    if ws.numel() < nbytes:
        raise ValueError(f"split workspace of {ws.numel()} bytes < {nbytes} required")
    N.check(lib.art_split_level(C.byref(prob), C.byref(prm), C.byref(res), ptr(ws), ws.numel(),
                                stream_handle(stream)), "art_split_level")
    out._keepalive = (x, y, ro, xo, dims_t, feats, temp, rid, pl, fb, th0, nk, ms)
    return out


def _level_result(K, R, M, max_dim, max_features, traces, dev) -> LevelResult:
    t = torch()
    out = LevelResult(
        theta=t.full((K, max_dim + 1), float("nan"), dtype=t.float64, device=dev),
        beta=t.full((K, 2, max_features), float("nan"), dtype=t.float64, device=dev),
        loss=t.empty(K, dtype=t.float64, device=dev),
        child_loss=t.empty((K, 2), dtype=t.float64, device=dev),
        ridge_effective=t.empty((K, 2), dtype=t.float64, device=dev),
        n_right=t.empty(K, dtype=t.int32, device=dev), n_iters=t.empty(K, dtype=t.int32, device=dev),
        stop_reason=t.empty(K, dtype=t.int32, device=dev), failure=t.empty(K, dtype=t.int32, device=dev),
        flags=t.empty(K, dtype=t.int32, device=dev), fallback_iteration=t.empty(K, dtype=t.int32, device=dev),
        final_alpha=t.empty(K, dtype=t.float64, device=dev))
    if traces:
        out.trace_loss = t.full((K, R, M + 1), float("nan"), dtype=t.float64, device=dev)
        out.trace_grad_norm = t.full((K, R, M + 1), float("nan"), dtype=t.float64, device=dev)
        out.trace_step = t.full((K, R, max(M, 1)), float("nan"), dtype=t.float64, device=dev)
        out.trace_backtracks = t.full((K, R, max(M, 1)), -1, dtype=t.int32, device=dev)
    return out


@dataclass
class SoftObliqueSplitter:
    """Soft sigmoid oblique splitter optimised by projected gradient descent on the GPU."""

    model_template: WeightedRegressionModel
    temperature: float
    max_iters: int = 100
    grad_atol: float = 1e-8
    grad_rtol: float = 1e-5
    min_side_points: int = 1
    min_side_fraction: float = 0.05
    min_side_fallback: bool = False
    n_restarts: int = 1
    alpha0: float = 1.0
    rho: float = 0.5
    armijo_c: float = 1e-4
    max_backtracks: int = 25
    adaptive_alpha: bool = True
    alpha_min: float = 1e-12
    alpha_max: float = 1e3
    alpha_grow: float = 10.0
    alpha_recovery: float = 10.0
    heavy_backtrack_threshold: int = 8
    max_line_search_failures: int = 3
    weight_floor: float = 1e-12
    refit_during_line_search: bool = False
    random_state: int | np.random.Generator | None = None
    split_timing_profile: SplitterTimingProfile | None = field(default=None, repr=False, compare=False)
    _timing_profile: BuildTimingProfile | None = field(default=None, init=False, repr=False)
    optimizer: Optimizer = "b200"
    backtrack_batch_size: int = 8
    qr_parallel: bool = True
    Xw_refresh: int = 32
    precision: Literal["fp64", "mixed"] = "fp64"
    tensor_gram: bool = False

    def _validate_inputs(self, X: np.ndarray, y: np.ndarray) -> None:
        """splitters.py:732-750"""

        if X.ndim != 2:
            raise ValueError(f"X must have shape (n, d), got {X.shape}.")
        if X.shape[0] != y.shape[0]:
            raise ValueError(f"X and y length mismatch: {X.shape[0]} != {y.shape[0]}.")
        if self.temperature <= 0.0:
            raise ValueError("temperature must be positive.")
        if self.max_iters < 0:
            raise ValueError("max_iters must be nonnegative.")
        if self.grad_atol < 0.0 or self.grad_rtol < 0.0:
            raise ValueError("gradient tolerances must be nonnegative.")
        if self.min_side_points < 1:
            raise ValueError("min_side_points must be at least 1.")
        if not (0.0 <= self.min_side_fraction < 0.5):
            raise ValueError("min_side_fraction must satisfy 0 <= fraction < 0.5.")
        if self.max_line_search_failures < 1:
            raise ValueError("max_line_search_failures must be at least 1.")
        if self.refit_during_line_search:
            raise ValueError("the GPU split search evaluates line-search candidates with frozen models.")

    def _required_side_points(self, n_total: int) -> int:
        return max(int(self.min_side_points), int(np.ceil(self.min_side_fraction * n_total)))

    def _rng(self) -> np.random.Generator:
        if isinstance(self.random_state, np.random.Generator):
            return self.random_state
        return np.random.default_rng(self.random_state)

    def _initialize_theta(self, X: np.ndarray, rng: np.random.Generator) -> np.ndarray:
        """splitters.py:692-700 (host draws, so restarts match the reference's stream)."""

        w = rng.normal(size=X.shape[1])
        nrm = np.linalg.norm(w)
        if nrm <= 1e-12:
            w[0] = 1.0
            nrm = 1.0
        w = w / nrm
        return np.concatenate([w, [float(np.median(X @ w))]])

    def split(self, X: np.ndarray, y: np.ndarray, parent_model: RegressionModel | None = None,
              parent_loss: float | None = None, prepared_design: PreparedDesign | None = None, *,
              hard_refit: bool = True, **unused) -> SplitResult:
        X = np.asarray(X, dtype=float)
        y = np.asarray(y, dtype=float).reshape(-1)
        self._validate_inputs(X, y)
        if not hard_refit and self.n_restarts != 1:
            raise ValueError("Skipping hard refits requires n_restarts == 1.")
        kind = _model_kind(self.model_template)
        rng = self._rng()
        if parent_model is None or parent_loss is None:
            pm = parent_model if parent_model is not None else self.model_template.clone().fit(X, y)
            parent_loss = mean_squared_error(y, pm.predict(X)) if parent_loss is None else parent_loss
            parent_model = pm
        R = max(1, self.n_restarts)
        theta0 = np.stack([self._initialize_theta(X, rng) for _ in range(R)])[None]
        res = split_level(self, X.reshape(-1), y, [0, X.shape[0]], [X.shape[1]], [kind], self.temperature,
                          self.model_template.ridge, parent_loss=[float(parent_loss)], theta0=theta0,
                          hard_refit=hard_refit, traces=True)
        return level_result_to_split(self, res, 0, X.shape[0], float(parent_loss), hard_refit)

    def split_temperatures(self, X: np.ndarray, y: np.ndarray, temperatures, parent_model: RegressionModel,
                           parent_loss: float, *, hard_refit: bool = True) -> list:
        """``split`` at several temperatures in one device launch.

        Entry i is what ``split`` returns with ``temperature = temperatures[i]``
        and this splitter's random state (the same restart starts for every
        temperature), or the SplitNotFoundError it raises.  The candidates
        run as nodes of one level over copies of the rows; a node's result
        does not depend on the other nodes of its level, so each entry is
        bit-identical to its own ``split`` call.
        """

        X = np.asarray(X, dtype=float)
        y = np.asarray(y, dtype=float).reshape(-1)
        self._validate_inputs(X, y)
        if not hard_refit and self.n_restarts != 1:
            raise ValueError("Skipping hard refits requires n_restarts == 1.")
        temps = np.asarray(temperatures, dtype=float).reshape(-1)
        K, (n, d) = temps.size, X.shape
        if K == 0:
            return []
        kind = _model_kind(self.model_template)
        rng = self._rng()
        R = max(1, self.n_restarts)
        theta0 = np.stack([self._initialize_theta(X, rng) for _ in range(R)])[None]
        # each candidate node holds its own copy of the rows: launches take at
        # most TEMPERATURE_BATCH_BYTES of copies (at least one candidate each)
        per = max(1, int(TEMPERATURE_BATCH_BYTES // max(1, n * (d + 1) * 8)))
        out = []
        for c0 in range(0, K, per):
            c = temps[c0:c0 + per]
            Kc = c.size
            res = split_level(self, np.tile(X.reshape(-1), Kc), np.tile(y, Kc), np.arange(Kc + 1) * n, [d] * Kc,
                              [kind] * Kc, c, self.model_template.ridge, parent_loss=[float(parent_loss)] * Kc,
                              theta0=np.repeat(theta0, Kc, axis=0), hard_refit=hard_refit, traces=True)
            for k in range(Kc):
                try:
                    out.append(level_result_to_split(self, res, k, n, float(parent_loss), hard_refit))
                except SplitNotFoundError as exc:
                    out.append(exc)
        return out


def level_result_to_split(s: SoftObliqueSplitter, res: LevelResult, k: int, n: int, parent_loss: float,
                          hard_refit: bool) -> SplitResult:
    """Export node k of a level result as a SplitResult, or raise SplitNotFoundError."""

    host = _host_level(res, k)
    d = int(np.count_nonzero(~np.isnan(host["theta"]))) - 1
    theta = host["theta"][: d + 1]
    reason = N.STOP_REASONS[host["stop_reason"]]
    failure = N.SPLIT_FAILURES[host["failure"]] if host["failure"] < len(N.SPLIT_FAILURES) else "invalid_split"
    pick = host["flags"] >> 8
    meta = {
        "optimizer": "b200", "n_iters": host["n_iters"], "stop_reason": reason,
        "converged": bool(host["flags"] & 1), "final_alpha": host["final_alpha"],
        "temperature": s.temperature, "restart": pick, "hard_refit": hard_refit,
        "required_side_points": s._required_side_points(n),
        # splitters.py:567-572
        "alpha_min_saturated": bool(s.adaptive_alpha and host["final_alpha"] <= s.alpha_min),
        "alpha_max_saturated": bool(s.adaptive_alpha and host["final_alpha"] >= s.alpha_max),
    }
    if res.trace_loss is not None:
        it = host["n_iters"]
        meta["soft_loss_history"] = host["trace_loss"][pick][: it + 1].tolist()
        meta["projected_grad_norm_history"] = host["trace_grad_norm"][pick][: it + 1].tolist()
        meta["step_size_history"] = host["trace_step"][pick][:it].tolist()
        meta["backtrack_history"] = [int(v) for v in host["trace_backtracks"][pick][:it]]
    if host["flags"] & 2:
        meta["min_side_fallback"] = True
        meta["fallback_iteration"] = host["fallback_iteration"]
    if failure is not None:
        meta["stop_reason"] = failure
        raise SplitNotFoundError(failure, f"GPU split search failed: {failure}", diagnostics=meta)
    n_right = host["n_right"]
    n_left = n - n_right
    meta.update(n_left=n_left, n_right=n_right)
    if not hard_refit:
        return SplitResult(w=theta[:-1].copy(), z=float(theta[-1]), left_model=None, right_model=None, loss=None,
                           parent_loss=parent_loss, split_gain=None, relative_split_gain=None, n_left=n_left,
                           n_right=n_right, converged=meta["converged"], n_iters=meta["n_iters"],
                           stop_reason=reason, metadata=meta)
    p = kind_feature_count(d, _model_kind(s.model_template))
    left = _clone_with(s.model_template, host["beta"][0, :p], host["ridge_effective"][0])
    right = _clone_with(s.model_template, host["beta"][1, :p], host["ridge_effective"][1])
    if isinstance(left, PolynomialRidgeModel):
        left._set_transformer(d)
        right._set_transformer(d)
    loss = float(host["loss"])
    meta.update(left_loss=float(host["child_loss"][0]), right_loss=float(host["child_loss"][1]))
    gain = parent_loss - loss
    return SplitResult(w=theta[:-1].copy(), z=float(theta[-1]), left_model=left, right_model=right, loss=loss,
                       parent_loss=parent_loss, split_gain=gain, relative_split_gain=gain / max(parent_loss, 1e-12),
                       n_left=n_left, n_right=n_right, converged=meta["converged"], n_iters=meta["n_iters"],
                       stop_reason=reason, metadata=meta)


def _host_level(res: LevelResult, k: int) -> dict:
    out = {}
    for name in ("theta", "beta", "loss", "child_loss", "ridge_effective", "n_right", "n_iters", "stop_reason",
                 "failure", "flags", "fallback_iteration", "final_alpha", "trace_loss", "trace_step",
                 "trace_backtracks", "trace_grad_norm"):
        v = getattr(res, name)
        if v is None:
            continue
        cache = getattr(res, "_host_cache", None)
        if cache is None:
            cache = {}
            res._host_cache = cache
        if name not in cache:
            cache[name] = v.cpu().numpy()
        val = cache[name][k]
        out[name] = val.item() if np.ndim(val) == 0 else val
    return out
