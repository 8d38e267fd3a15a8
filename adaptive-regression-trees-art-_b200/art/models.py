"""Weighted ridge models whose solves run on the B200 kernels.

Public names and semantics follow the reference ``art/models.py``:
``solve_weighted_ridge`` (models.py:218-371), ``AffineRidgeModel``
(472-554, bias last), ``PolynomialRidgeModel`` (557-694, sklearn order, bias
first), ``RidgeSolveResult`` (25-36), ``PreparedDesign`` (85-119),
``scaled_ridge_from_gram`` (209-215).  Every fit is one launch sequence of
``art_ridge_batched``; ``solve_weighted_ridge_batched`` exposes the batched
form on device tensors directly.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from math import comb
from typing import Callable, Literal, Protocol, runtime_checkable

import numpy as np

from . import _native as N
from ._device import WORKSPACES, ptr, require_cuda, stream_handle, to_device, torch

RidgeSolver = Literal["auto", "normal", "qr", "svd"]
ResolvedRidgeSolver = Literal["cholesky", "qr", "svd"]
ConditionEstimator = Literal[
    "sqrt_gram_1norm", "svd_2norm", "cholesky_failure", "condition_estimate_failure"
]
RIDGE_SOLVERS: tuple[RidgeSolver, ...] = ("auto", "normal", "qr", "svd")
DEFAULT_AUTO_RCOND_THRESHOLD = 1e-10
MODEL_CONDITION_WARNING_THRESHOLD = 1e10
Precision = Literal["fp64", "mixed"]
_SOLVER_CODES = {"normal": N.SOLVER_NORMAL, "auto": N.SOLVER_AUTO, "qr": N.SOLVER_QR, "svd": N.SOLVER_SVD}
_PRECISION_CODES = {"fp64": N.PRECISION_FP64, "mixed": N.PRECISION_MIXED}


@dataclass(frozen=True)
class RidgeSolveResult:
    """Coefficients and numerical diagnostics from one ridge solve."""

    coefficients: np.ndarray
    solver_requested: RidgeSolver
    solver_used: ResolvedRidgeSolver
    condition_estimator: ConditionEstimator | None
    cond_estimate: float | None
    ridge_effective: float
    rank: int | None = None
    fallback_reason: str | None = None


@dataclass(frozen=True)
class WeightedNormalEquations:
    """Precomputed normal equations (kept for API compatibility).

    The B200 kernels form Grams on chip from the raw rows, so a precomputed
    system is not accepted by :func:`solve_weighted_ridge`.
    """

    gram: np.ndarray
    rhs: np.ndarray
    subtraction_bound: float = 0.0
    rebuild: Callable[[], "WeightedNormalEquations"] | None = field(
        default=None, repr=False, compare=False
    )
    subtraction_rhs_bound: float = 0.0


@runtime_checkable
class RegressionModel(Protocol):
    def fit(self, X: np.ndarray, y: np.ndarray) -> "RegressionModel": ...

    def predict(self, X: np.ndarray) -> np.ndarray: ...

    def clone(self) -> "RegressionModel": ...


@runtime_checkable
class WeightedRegressionModel(RegressionModel, Protocol):
    def fit_weighted(
        self, X: np.ndarray, y: np.ndarray, weights: np.ndarray, weight_floor: float = 1e-12
    ) -> "WeightedRegressionModel": ...


@dataclass(frozen=True)
class PreparedDesign:
    """Feature matrix and fitted transform state for one ordered sample set."""

    matrix: np.ndarray
    input_dimension: int
    feature_signature: tuple[object, ...]
    feature_state: object

    def __post_init__(self) -> None:
        matrix = np.asarray(self.matrix, dtype=float)
        if matrix.ndim != 2:
            raise ValueError(f"Prepared design matrix must have shape (n, p), got {matrix.shape}.")
        if self.input_dimension < 1:
            raise ValueError("Prepared design input_dimension must be at least 1.")
        object.__setattr__(self, "matrix", matrix)

    @property
    def n_samples(self) -> int:
        return self.matrix.shape[0]

    def subset(self, rows: np.ndarray) -> "PreparedDesign":
        matrix = self.matrix[rows]
        if matrix.ndim == 1:
            matrix = matrix.reshape(1, -1)
        return PreparedDesign(matrix, self.input_dimension, self.feature_signature, self.feature_state)


@runtime_checkable
class PreparedFeatureModel(WeightedRegressionModel, Protocol):
    def prepare_design(self, X: np.ndarray) -> PreparedDesign: ...

    def fit_design(self, prepared: PreparedDesign, y: np.ndarray) -> "PreparedFeatureModel": ...

    def fit_weighted_design(
        self, prepared: PreparedDesign, y: np.ndarray, weights: np.ndarray, weight_floor: float = 1e-12
    ) -> "PreparedFeatureModel": ...

    def predict_design(self, prepared: PreparedDesign) -> np.ndarray: ...


def polynomial_feature_count(input_dimension: int, degree: int, include_bias: bool = True) -> int:
    input_dimension, degree = int(input_dimension), int(degree)
    if input_dimension < 1:
        raise ValueError("input_dimension must be at least 1.")
    if degree < 1:
        raise ValueError("degree must be at least 1.")
    count = comb(input_dimension + degree, degree)
    return count if include_bias else count - 1


def model_effective_dimension(model: RegressionModel, input_dimension: int) -> int:
    method = getattr(model, "effective_dimension", None)
    if method is None:
        raise TypeError(
            f"{type(model).__name__} does not define effective_dimension; "
            "provide an explicit sample_count policy to the tree builder."
        )
    dimension = int(method(input_dimension))
    if dimension < 1:
        raise ValueError("Model effective_dimension must be at least 1.")
    return dimension


def ridge_solve_diagnostics(model: object) -> dict[str, object] | None:
    result = model if isinstance(model, RidgeSolveResult) else getattr(model, "solve_result_", None)
    if not isinstance(result, RidgeSolveResult):
        return None
    return {
        "solver_requested": result.solver_requested,
        "solver_used": result.solver_used,
        "condition_estimator": result.condition_estimator,
        "cond_estimate": result.cond_estimate,
        "ridge_effective": result.ridge_effective,
        "rank": result.rank,
        "fallback_reason": result.fallback_reason,
    }


def augment_features(X: np.ndarray) -> np.ndarray:
    X = np.asarray(X, dtype=float)
    if X.ndim == 1:
        X = X.reshape(1, -1)
    if X.ndim != 2:
        raise ValueError(f"X must have shape (n, d), got {X.shape}.")
    return np.hstack([X, np.ones((X.shape[0], 1))])


def scaled_ridge_from_gram(gram: np.ndarray, ridge: float) -> float:
    """Scale ridge by the mean eigenvalue of the Gram matrix."""

    gram = np.asarray(gram, dtype=float)
    if gram.ndim != 2 or gram.shape[0] != gram.shape[1]:
        raise ValueError(f"gram must be square, got {gram.shape}.")
    return float(ridge) * float(np.trace(gram)) / gram.shape[0]


def feature_kind(degree: int, include_bias: bool, bias_last: bool = False) -> int:
    """Map a model's feature basis to the kernel's ART_FEATURES_* code."""

    if bias_last:
        if degree != 1 or not include_bias:
            raise ValueError("bias-last features are affine only")
        return N.FEATURES_AFFINE
    if degree == 1:
        return N.FEATURES_POLY1 if include_bias else N.FEATURES_POLY1_NOBIAS
    if degree == 2:
        return N.FEATURES_POLY2 if include_bias else N.FEATURES_POLY2_NOBIAS
    raise ValueError("on-chip features support degree 1 or 2")


def kind_feature_count(d: int, kind: int) -> int:
    if kind in (N.FEATURES_AFFINE, N.FEATURES_POLY1):
        return d + 1
    if kind == N.FEATURES_POLY1_NOBIAS:
        return d
    if kind == N.FEATURES_POLY2:
        return 1 + d + d * (d + 1) // 2
    if kind == N.FEATURES_POLY2_NOBIAS:
        return d + d * (d + 1) // 2
    raise ValueError(f"unknown feature kind {kind}")


# ---------------------------------------------------------------- batched
@dataclass
class BatchedRidgeResult:
    """Device outputs of one batched solve (torch CUDA tensors)."""

    beta: object            # (K, beta_stride) float64
    ridge_effective: object  # (K,) float64
    cond_estimate: object | None
    status: object          # (K,) int32
    info: object            # (K,) int32 (ART_INFO_* bits)


def _factor_choice(requested, precision) -> bool:
    """Explicit FP64-factorisation flag, else the autotuner's cached choice, else FP32."""

    if requested is not None:
        return bool(requested)
    if precision != "mixed":
        return False
    from . import autotune

    return bool(autotune.cached_ridge_choice()[1])


def _tensor_threshold(requested, precision, dims_t, feats, ro, max_features) -> int:
    """Explicit threshold, else the autotuner's cached choice, else 0 (library default)."""

    if requested is not None:
        return int(requested)
    if precision != "mixed":
        return 0
    from . import autotune

    return autotune.cached_ridge_choice()[0]


def solve_weighted_ridge_batched(
    x,
    y,
    weights,
    row_offsets,
    dims,
    features,
    ridge,
    *,
    x_offsets=None,
    weight_floor: float = 1e-12,
    solver: RidgeSolver = "normal",
    precision: Precision = "fp64",
    auto_rcond_threshold: float = DEFAULT_AUTO_RCOND_THRESHOLD,
    max_features: int | None = None,
    max_dim: int | None = None,
    condition: bool = False,
    fp64_factor: bool | None = None,
    tensor_min_features: int | None = None,
    out: BatchedRidgeResult | None = None,
    stream=None,
    host_slices: int | None = None,
) -> BatchedRidgeResult:
    """Solve K weighted ridge systems in one stream-ordered launch sequence.

    ``x`` holds each system's (n_k, d_k) rows row-major at ``x_offsets[k]``
    (default: ``row_offsets[k] * d_k`` for uniform d); ``y``/``weights`` hold
    one value per row, system k owning rows ``row_offsets[k]:row_offsets[k+1]``.
    ``weights=None`` means unit weights.  All array arguments may be numpy or
    torch; they are moved to the current CUDA device.  No host sync happens
    unless the caller reads the result.  ``fp64_factor`` makes the mixed form
    factor its tensor-core Gram in FP64 (``ART_RIDGE_OPT_FP64_FACTOR``); None
    takes the autotuned choice for this device, else FP32.
    ``tensor_min_features`` is the smallest feature count the mixed form
    solves on the tensor cores (smaller systems take the FP64 kernels); None
    takes the autotuned choice for this device and batch, else the library
    default (33).
    ``host_slices``: when ``x`` is in host memory (numpy, or a CPU tensor;
    pinned for the copies to run asynchronously) and the systems' rows are
    stored back to back, the batch is cut into this many slices of
    contiguous systems of about equal rows.  Each slice's host-to-device
    copy runs on a side stream while the previous slice is solved, so the
    copies and the solves overlap.  None picks 8 for host inputs of at least
    64 MB and 1 (one copy, then one solve) otherwise.  Results do not depend
    on the slicing.
    """

    t = torch()
    lib = N.load_library()
    dev = require_cuda()
    slices = host_slices
    on_host = isinstance(x, np.ndarray) or (isinstance(x, t.Tensor) and x.device.type == "cpu")
    if slices is None:
        nbytes_x = int(x.nbytes) if isinstance(x, np.ndarray) else (int(x.numel() * x.element_size()) if on_host else 0)
        slices = 8 if on_host and nbytes_x >= (64 << 20) else 1
    if on_host and int(slices) > 1:
        staged = _solve_host_staged(
            x, y, weights, row_offsets, dims, features, ridge, x_offsets, int(slices), stream,
            dict(weight_floor=weight_floor, solver=solver, precision=precision,
                 auto_rcond_threshold=auto_rcond_threshold, max_features=max_features, max_dim=max_dim,
                 condition=condition, fp64_factor=fp64_factor, tensor_min_features=tensor_min_features),
            out)
        if staged is not None:
            return staged
    if solver not in _SOLVER_CODES:
        raise ValueError(f"solver must be one of {RIDGE_SOLVERS}, got {solver!r}.")
    if precision not in _PRECISION_CODES:
        raise ValueError("precision must be 'fp64' or 'mixed'.")
    if not np.isfinite(auto_rcond_threshold) or not (0.0 < auto_rcond_threshold <= 1.0):
        raise ValueError("auto_rcond_threshold must satisfy 0 < value <= 1.")
    x = to_device(x, t.float64, dev)
    y = to_device(y, t.float64, dev)
    w = None if weights is None else to_device(weights, t.float64, dev)
    ro = to_device(row_offsets, t.int64, dev)
    dims_t = to_device(dims, t.int32, dev)
    feats = to_device(features, t.int32, dev)
    K = int(dims_t.numel())
    ridge_t = to_device(np.broadcast_to(np.asarray(ridge, dtype=float), (K,)) if not isinstance(ridge, t.Tensor) else ridge, t.float64, dev)
    if ridge_t.numel() == 1 and K != 1:
        ridge_t = ridge_t.expand(K).contiguous()
    if x_offsets is None:
        x_offsets = ro[:-1] * dims_t.to(t.int64)
    xo = to_device(x_offsets, t.int64, dev)
    if max_features is None or max_dim is None:
        dh = dims_t.cpu().numpy()
        fh = feats.cpu().numpy()
        if max_dim is None:
            max_dim = int(dh.max()) if K else 1
        if max_features is None:
            max_features = max((kind_feature_count(int(d), int(f)) for d, f in zip(dh, fh)), default=1)
    if max_features > N.MAX_FEATURES:
        raise ValueError(f"at most {N.MAX_FEATURES} features per system are supported")
    if out is None:
        stride = int(max_features)
        out = BatchedRidgeResult(
            beta=t.full((K, stride), float("nan"), dtype=t.float64, device=dev),
            ridge_effective=t.empty(K, dtype=t.float64, device=dev),
            cond_estimate=t.empty(K, dtype=t.float64, device=dev) if (condition or solver == "auto") else None,
            status=t.empty(K, dtype=t.int32, device=dev),
            info=t.empty(K, dtype=t.int32, device=dev),
        )
    seg = N.ArtSegments(K, ptr(ro), ptr(xo), ptr(dims_t), ptr(feats))
    prob = N.ArtRidgeProblem(
        seg, ptr(x), ptr(y), ptr(w), ptr(ridge_t), float(weight_floor), _SOLVER_CODES[solver],
        _PRECISION_CODES[precision], float(auto_rcond_threshold), int(max_features), int(max_dim),
        N.RIDGE_OPT_FP64_FACTOR if _factor_choice(fp64_factor, precision) else 0,
        int(_tensor_threshold(tensor_min_features, precision, dims_t, feats, ro, max_features)),
    )
    res = N.ArtRidgeResult(
        ptr(out.beta), int(out.beta.shape[1]), ptr(out.ridge_effective), ptr(out.cond_estimate),
        ptr(out.status), ptr(out.info),
    )
    nbytes = lib.art_ridge_workspace_size(K, int(max_features))
    ws = WORKSPACES.get(nbytes, stream)
    rc = lib.art_ridge_batched(C.byref(prob), C.byref(res), ptr(ws), ws.numel(), stream_handle(stream))
    N.check(rc, "art_ridge_batched")
    # keep inputs alive until the stream has consumed them
    out._keepalive = (x, y, w, ro, xo, dims_t, feats, ridge_t)
    return out


_COPY_STREAMS: dict[int, object] = {}


def _host_f64(a, t):
    """numpy / torch CPU array -> contiguous float64 CPU tensor (no copy when already suitable)."""

    if isinstance(a, t.Tensor):
        return a.to(dtype=t.float64).contiguous()
    return t.from_numpy(np.ascontiguousarray(a, dtype=np.float64))


def host_slice_bounds(row_offsets, x_offsets, dims, slices: int):
    """System boundaries [0, k1, ..., K] of up to ``slices`` slices with about
    equal rows, or None when the layout cannot be staged in slices: fewer
    than two systems, or rows / x blocks not stored back to back from 0."""

    ro = np.asarray(row_offsets, dtype=np.int64)
    xo = np.asarray(x_offsets, dtype=np.int64)
    d = np.asarray(dims, dtype=np.int64)
    K = int(d.size)
    if K < 2 or slices < 2 or ro.size != K + 1 or xo.size != K:
        return None
    ends = xo + np.diff(ro) * d
    if ro[0] != 0 or xo[0] != 0 or np.any(np.diff(ro) < 0) or not np.array_equal(xo[1:], ends[:-1]):
        return None
    cuts = np.searchsorted(ro, np.linspace(0, ro[-1], slices + 1)[1:-1], side="left")
    return np.unique(np.concatenate([[0], np.clip(cuts, 1, K - 1), [K]])).astype(np.int64)


def _solve_host_staged(x, y, weights, row_offsets, dims, features, ridge, x_offsets, slices, stream, kw, out):
    """Overlapped host-to-device staging for solve_weighted_ridge_batched.

    Returns None (the caller then copies everything at once) when the
    systems' rows and x blocks are not stored back to back from offset 0.
    """

    t = torch()
    dev = require_cuda()
    ro_h = np.asarray(row_offsets.cpu() if isinstance(row_offsets, t.Tensor) else row_offsets, dtype=np.int64)
    dims_h = np.asarray(dims.cpu() if isinstance(dims, t.Tensor) else dims, dtype=np.int64)
    feats_h = np.asarray(features.cpu() if isinstance(features, t.Tensor) else features, dtype=np.int32)
    K = int(dims_h.size)
    if ro_h.size != K + 1:
        return None
    xo_h = (ro_h[:-1] * dims_h if x_offsets is None else
            np.asarray(x_offsets.cpu() if isinstance(x_offsets, t.Tensor) else x_offsets, dtype=np.int64))
    bounds = host_slice_bounds(ro_h, xo_h, dims_h, slices)
    if bounds is None:
        return None
    ends = xo_h + np.diff(ro_h) * dims_h
    xh = _host_f64(x, t)
    yh = _host_f64(y, t)
    wh = None if weights is None else _host_f64(weights, t)
    if xh.numel() < int(ends[-1]) or yh.numel() < int(ro_h[-1]) or (wh is not None and wh.numel() < int(ro_h[-1])):
        raise ValueError("x, y and weights must cover every system's rows")
    if kw.get("max_dim") is None:
        kw["max_dim"] = int(dims_h.max())
    if kw.get("max_features") is None:
        kw["max_features"] = max(kind_feature_count(int(d), int(f)) for d, f in zip(dims_h, feats_h))
    comp = t.cuda.current_stream(dev) if stream is None else stream
    copy = _COPY_STREAMS.get(dev.index)
    if copy is None:
        copy = _COPY_STREAMS[dev.index] = t.cuda.Stream(device=dev)
    with t.cuda.stream(comp):
        xd = t.empty(xh.numel(), dtype=t.float64, device=dev)
        yd = t.empty(yh.numel(), dtype=t.float64, device=dev)
        wd = None if wh is None else t.empty(wh.numel(), dtype=t.float64, device=dev)
        ro_d = t.from_numpy(ro_h).to(dev)
        xo_d = t.from_numpy(xo_h).to(dev)
        dims_d = t.from_numpy(dims_h.astype(np.int32)).to(dev)
        feats_d = t.from_numpy(feats_h).to(dev)
        ridge_d = to_device(np.broadcast_to(np.asarray(ridge, dtype=float), (K,)).copy()
                            if not isinstance(ridge, t.Tensor) else ridge, t.float64, dev)
        if ridge_d.numel() == 1:
            ridge_d = ridge_d.expand(K).contiguous()
        if out is None:
            pm = int(kw["max_features"])
            cond = kw.get("condition") or kw.get("solver") == "auto"
            out = BatchedRidgeResult(
                beta=t.full((K, pm), float("nan"), dtype=t.float64, device=dev),
                ridge_effective=t.empty(K, dtype=t.float64, device=dev),
                cond_estimate=t.empty(K, dtype=t.float64, device=dev) if cond else None,
                status=t.empty(K, dtype=t.int32, device=dev),
                info=t.empty(K, dtype=t.int32, device=dev),
            )
    for buf in (xd, yd, wd):
        if buf is not None:
            buf.record_stream(copy)
    copy.wait_stream(comp)
    pinned = xh.is_pinned()
    for k0, k1 in zip(bounds[:-1].tolist(), bounds[1:].tolist()):
        r0, r1, e0, e1 = int(ro_h[k0]), int(ro_h[k1]), int(xo_h[k0]), int(ends[k1 - 1])
        with t.cuda.stream(copy):
            xd[e0:e1].copy_(xh[e0:e1], non_blocking=pinned)
            yd[r0:r1].copy_(yh[r0:r1], non_blocking=pinned)
            if wd is not None:
                wd[r0:r1].copy_(wh[r0:r1], non_blocking=pinned)
            ev = t.cuda.Event()
            ev.record(copy)
        comp.wait_event(ev)
        part = BatchedRidgeResult(
            beta=out.beta[k0:k1], ridge_effective=out.ridge_effective[k0:k1],
            cond_estimate=None if out.cond_estimate is None else out.cond_estimate[k0:k1],
            status=out.status[k0:k1], info=out.info[k0:k1])
        solve_weighted_ridge_batched(xd, yd, wd, ro_d[k0:k1 + 1], dims_d[k0:k1], feats_d[k0:k1], ridge_d[k0:k1],
                                     x_offsets=xo_d[k0:k1], out=part, stream=comp, host_slices=1, **kw)
    # the host buffers must outlive the queued copies
    out._keepalive = (xh, yh, wh, xd, yd, wd, ro_d, xo_d, dims_d, feats_d, ridge_d)
    return out


def ridge_gram_batched(x, y, weights, row_offsets, dims, features, *, x_offsets=None,
                       weight_floor: float = 1e-12, max_features: int | None = None,
                       max_dim: int | None = None, stream=None):
    """Tensor-core weighted Grams (TF32 hi/lo split products, FP32 accumulation).

    Returns (packed lower-triangular Grams [K, pmax(pmax+1)/2] float32, status[K]);
    systems outside 33 <= p <= 160 get status -4.
    """

    t = torch()
    lib = N.load_library()
    dev = require_cuda()
    x = to_device(x, t.float64, dev)
    y = to_device(y, t.float64, dev)
    w = None if weights is None else to_device(weights, t.float64, dev)
    ro = to_device(row_offsets, t.int64, dev)
    dims_t = to_device(dims, t.int32, dev)
    feats = to_device(features, t.int32, dev)
    K = int(dims_t.numel())
    if x_offsets is None:
        x_offsets = ro[:-1] * dims_t.to(t.int64)
    xo = to_device(x_offsets, t.int64, dev)
    if max_features is None:
        max_features = max(kind_feature_count(int(d), int(f)) for d, f in zip(dims_t.cpu().numpy(), feats.cpu().numpy()))
    if max_dim is None:
        max_dim = int(dims_t.max().item())
    ridge_t = t.zeros(K, dtype=t.float64, device=dev)
    E = max_features * (max_features + 1) // 2
    gram = t.full((K, E), float("nan"), dtype=t.float32, device=dev)
    status = t.empty(K, dtype=t.int32, device=dev)
    seg = N.ArtSegments(K, ptr(ro), ptr(xo), ptr(dims_t), ptr(feats))
    prob = N.ArtRidgeProblem(seg, ptr(x), ptr(y), ptr(w), ptr(ridge_t), float(weight_floor), N.SOLVER_NORMAL,
                             N.PRECISION_MIXED, 1e-10, int(max_features), int(max_dim), 0, 0)
    nbytes = lib.art_ridge_workspace_size(K, int(max_features))
    ws = WORKSPACES.get(nbytes, stream)
    rc = lib.art_ridge_gram(C.byref(prob), ptr(gram), E, ptr(status), ptr(ws), ws.numel(), stream_handle(stream))
    N.check(rc, "art_ridge_gram")
    gram._keepalive = (x, y, w, ro, xo, dims_t, feats, ridge_t)
    return gram, status


# ---------------------------------------------------------------- single
def _result_from_row(beta, ridge_eff, cond, status, info, p, solver) -> RidgeSolveResult:
    fallback = None
    solver_used: ResolvedRidgeSolver = "cholesky"
    estimator: ConditionEstimator | None = None
    cond_estimate: float | None = None
    if info & N.INFO_SVD:
        # solver="svd", or auto whose QR solution was not finite (models.py:426-442)
        return RidgeSolveResult(
            coefficients=np.asarray(beta[:p], dtype=float).copy(), solver_requested=solver, solver_used="svd",
            condition_estimator="svd_2norm", cond_estimate=float(cond) if cond is not None else None,
            ridge_effective=float(ridge_eff), rank=(int(info) >> N.INFO_RANK_SHIFT) & 0xFF,
            fallback_reason="qr_nonfinite" if info & N.INFO_QR_FALLBACK else None)
    if info & N.INFO_QR_FALLBACK:
        solver_used = "qr"
        if info & N.INFO_CHOLESKY_FAILED:
            fallback, estimator, cond_estimate = "cholesky_failed", "cholesky_failure", float("inf")
        elif info & N.INFO_RCOND_BELOW:
            fallback, estimator = "rcond_below_threshold", "sqrt_gram_1norm"
            cond_estimate = float(cond)
    elif cond is not None:
        if info & N.INFO_COND_FAILED:
            estimator, cond_estimate = "condition_estimate_failure", float("inf")
        else:
            estimator, cond_estimate = "sqrt_gram_1norm", float(cond)
    return RidgeSolveResult(
        coefficients=np.asarray(beta[:p], dtype=float).copy(),
        solver_requested=solver,
        solver_used=solver_used,
        condition_estimator=estimator,
        cond_estimate=cond_estimate,
        ridge_effective=float(ridge_eff),
        rank=p if solver_used == "qr" else None,
        fallback_reason=fallback,
    )


def _solve_single(x, y, weights, ridge, kind, *, weight_floor, solver, auto_rcond_threshold,
                  precision="fp64") -> RidgeSolveResult:
    x = np.ascontiguousarray(x, dtype=float)
    y = np.asarray(y, dtype=float).reshape(-1)
    n, d = x.shape
    if y.shape[0] != n:
        raise ValueError("design, y, and weights must have the same number of rows.")
    if weights is not None:
        weights = np.asarray(weights, dtype=float).reshape(-1)
        if weights.shape[0] != n:
            raise ValueError("design, y, and weights must have the same number of rows.")
        if np.any(weights < 0.0):
            raise ValueError("weights must be nonnegative.")
    if ridge < 0.0:
        raise ValueError("ridge must be nonnegative.")
    p = kind_feature_count(d, kind)
    out = solve_weighted_ridge_batched(
        x if n else np.zeros((0, d)), y, weights, np.array([0, n], dtype=np.int64), [d], [kind], [float(ridge)],
        weight_floor=weight_floor, solver=solver, precision=precision,
        auto_rcond_threshold=auto_rcond_threshold, max_features=p, max_dim=d,
        condition=True,
    )
    beta = out.beta.cpu().numpy()[0]
    status = int(out.status.cpu().numpy()[0])
    info = int(out.info.cpu().numpy()[0])
    ridge_eff = float(out.ridge_effective.cpu().numpy()[0])
    cond = float(out.cond_estimate.cpu().numpy()[0]) if out.cond_estimate is not None else None
    if status > 0:
        raise np.linalg.LinAlgError(
            "Normal-equation Cholesky factorization failed; use solver='auto', "
            "solver='qr', or solver='svd', or increase ridge regularization."
        )
    if status in (-1, -2):
        raise ValueError("design, y and weights must be finite and weights nonnegative.")
    if status == -3:
        raise np.linalg.LinAlgError("Ridge solve produced non-finite coefficients.")
    if status < 0:
        raise RuntimeError(f"art_ridge_batched status {status}")
    return _result_from_row(beta, ridge_eff, cond, status, info, p, solver)


def solve_weighted_ridge(
    design: np.ndarray,
    y: np.ndarray,
    weights: np.ndarray,
    ridge: float,
    weight_floor: float = 1e-12,
    solver: RidgeSolver = "normal",
    auto_rcond_threshold: float = DEFAULT_AUTO_RCOND_THRESHOLD,
    *,
    normal_equations: WeightedNormalEquations | None = None,
) -> RidgeSolveResult:
    """GPU weighted, trace-scaled ridge solve of an explicit design matrix."""

    if normal_equations is not None:
        raise ValueError("Precomputed normal equations are not used by the B200 path.")
    design = np.asarray(design, dtype=float)
    if design.ndim != 2:
        raise ValueError(f"design must have shape (n, p), got {design.shape}.")
    if solver not in RIDGE_SOLVERS:
        raise ValueError(f"solver must be one of {RIDGE_SOLVERS}, got {solver!r}.")
    if not np.isfinite(auto_rcond_threshold) or not (0.0 < auto_rcond_threshold <= 1.0):
        raise ValueError("auto_rcond_threshold must satisfy 0 < value <= 1.")
    return _solve_single(design, y, weights, ridge, N.FEATURES_POLY1_NOBIAS,
                         weight_floor=weight_floor, solver=solver,
                         auto_rcond_threshold=auto_rcond_threshold)


def _validate_ridge_solver(solver: str) -> None:
    if solver not in RIDGE_SOLVERS:
        raise ValueError(f"solver must be one of {RIDGE_SOLVERS}, got {solver!r}.")


def _validate_auto_rcond_threshold(value: float) -> None:
    if not np.isfinite(value) or not (0.0 < value <= 1.0):
        raise ValueError("auto_rcond_threshold must satisfy 0 < value <= 1.")


# ---------------------------------------------------------------- models
@dataclass
class AffineRidgeModel:
    """Affine model ``[x, 1] @ coef`` fit by weighted ridge on the GPU."""

    ridge: float = 1e-8
    solver: RidgeSolver = "normal"
    auto_rcond_threshold: float = DEFAULT_AUTO_RCOND_THRESHOLD
    coef_: np.ndarray | None = field(default=None, init=False, repr=False)
    solve_result_: RidgeSolveResult | None = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        _validate_ridge_solver(self.solver)
        _validate_auto_rcond_threshold(self.auto_rcond_threshold)

    feature_kind = N.FEATURES_AFFINE

    def effective_dimension(self, input_dimension: int) -> int:
        input_dimension = int(input_dimension)
        if input_dimension < 1:
            raise ValueError("input_dimension must be at least 1.")
        return input_dimension + 1

    def kind(self, input_dimension: int | None = None) -> int:
        return N.FEATURES_AFFINE

    def fit(self, X: np.ndarray, y: np.ndarray) -> "AffineRidgeModel":
        X = _as_2d(X)
        y = np.asarray(y, dtype=float).reshape(-1)
        if X.shape[0] != y.shape[0]:
            raise ValueError(f"X and y length mismatch: {X.shape[0]} != {y.shape[0]}.")
        return self._fit(X, y, None, 1e-12)

    def fit_weighted(self, X, y, weights, weight_floor: float = 1e-12, *, normal_equations=None):
        if normal_equations is not None:
            raise ValueError("Precomputed normal equations are not used by the B200 path.")
        return self._fit(_as_2d(X), np.asarray(y, dtype=float).reshape(-1), weights, weight_floor)

    def _fit(self, X, y, weights, weight_floor):
        self.solve_result_ = _solve_single(
            X, y, weights, self.ridge, N.FEATURES_AFFINE, weight_floor=weight_floor,
            solver=self.solver, auto_rcond_threshold=self.auto_rcond_threshold,
        )
        self.coef_ = self.solve_result_.coefficients
        return self

    def predict(self, X: np.ndarray) -> np.ndarray:
        if self.coef_ is None:
            raise ValueError("Model must be fit before calling predict.")
        X = _as_2d(X)
        if X.shape[1] != self.coef_.shape[0] - 1:
            raise ValueError(f"X must have {self.coef_.shape[0] - 1} columns, got {X.shape[1]}.")
        return X @ self.coef_[:-1] + self.coef_[-1]

    def clone(self) -> "AffineRidgeModel":
        return AffineRidgeModel(ridge=self.ridge, solver=self.solver,
                                auto_rcond_threshold=self.auto_rcond_threshold)


@dataclass
class PolynomialRidgeModel:
    """Polynomial feature model (sklearn order) fit by weighted ridge on the GPU."""

    degree: int = 2
    ridge: float = 1e-8
    include_bias: bool = True
    solver: RidgeSolver = "normal"
    auto_rcond_threshold: float = DEFAULT_AUTO_RCOND_THRESHOLD
    transformer_: object | None = field(default=None, init=False, repr=False)
    coef_: np.ndarray | None = field(default=None, init=False, repr=False)
    solve_result_: RidgeSolveResult | None = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        from sklearn.preprocessing import PolynomialFeatures

        _validate_ridge_solver(self.solver)
        _validate_auto_rcond_threshold(self.auto_rcond_threshold)
        self.transformer_ = PolynomialFeatures(degree=self.degree, include_bias=self.include_bias)

    def effective_dimension(self, input_dimension: int) -> int:
        return polynomial_feature_count(input_dimension, self.degree, include_bias=self.include_bias)

    def kind(self, input_dimension: int | None = None) -> int:
        return feature_kind(self.degree, self.include_bias)

    def fit(self, X: np.ndarray, y: np.ndarray) -> "PolynomialRidgeModel":
        return self.fit_weighted(X, y, None)

    def fit_weighted(self, X, y, weights, weight_floor: float = 1e-12):
        X = _as_2d(X)
        y = np.asarray(y, dtype=float).reshape(-1)
        if self.degree in (1, 2):
            self.solve_result_ = _solve_single(
                X, y, weights, self.ridge, self.kind(), weight_floor=weight_floor,
                solver=self.solver, auto_rcond_threshold=self.auto_rcond_threshold,
            )
            self._set_transformer(X.shape[1])
            self.coef_ = self.solve_result_.coefficients
            return self
        return self.fit_weighted_design(self.prepare_design(X), y, weights, weight_floor)

    def _set_transformer(self, d: int) -> None:
        from sklearn.preprocessing import PolynomialFeatures

        transformer = PolynomialFeatures(degree=self.degree, include_bias=self.include_bias)
        transformer.fit(np.zeros((1, d)))
        self.transformer_ = transformer

    def prepare_design(self, X: np.ndarray) -> PreparedDesign:
        from sklearn.preprocessing import PolynomialFeatures

        X = _as_2d(X)
        transformer = PolynomialFeatures(degree=self.degree, include_bias=self.include_bias)
        return PreparedDesign(transformer.fit_transform(X), X.shape[1], self._feature_signature(), transformer)

    def fit_design(self, prepared: PreparedDesign, y: np.ndarray) -> "PolynomialRidgeModel":
        return self.fit_weighted_design(prepared, y, None)

    def fit_weighted_design(self, prepared, y, weights, weight_floor: float = 1e-12, *, normal_equations=None):
        if normal_equations is not None:
            raise ValueError("Precomputed normal equations are not used by the B200 path.")
        self._validate_prepared(prepared)
        self.solve_result_ = _solve_single(
            prepared.matrix, np.asarray(y, dtype=float).reshape(-1), weights, self.ridge,
            N.FEATURES_POLY1_NOBIAS, weight_floor=weight_floor, solver=self.solver,
            auto_rcond_threshold=self.auto_rcond_threshold,
        )
        self.transformer_ = prepared.feature_state
        self.coef_ = self.solve_result_.coefficients
        return self

    def predict(self, X: np.ndarray) -> np.ndarray:
        if self.coef_ is None:
            raise ValueError("Model must be fit before calling predict.")
        return self.transformer_.transform(np.asarray(X, dtype=float)) @ self.coef_

    def predict_design(self, prepared: PreparedDesign) -> np.ndarray:
        if self.coef_ is None:
            raise ValueError("Model must be fit before calling predict_design.")
        self._validate_prepared(prepared)
        if prepared.matrix.shape[1] != self.coef_.shape[0]:
            raise ValueError("Prepared design feature count does not match fitted coefficients.")
        return prepared.matrix @ self.coef_

    def clone(self) -> "PolynomialRidgeModel":
        return PolynomialRidgeModel(degree=self.degree, ridge=self.ridge, include_bias=self.include_bias,
                                    solver=self.solver, auto_rcond_threshold=self.auto_rcond_threshold)

    def _feature_signature(self) -> tuple[object, ...]:
        return ("polynomial", self.degree, self.include_bias)

    def _validate_prepared(self, prepared: PreparedDesign) -> None:
        if not isinstance(prepared, PreparedDesign):
            raise TypeError("prepared must be a PreparedDesign.")
        if prepared.feature_signature != self._feature_signature():
            raise ValueError("Prepared design does not match this polynomial model configuration.")
        expected = self.effective_dimension(prepared.input_dimension)
        if prepared.matrix.shape[1] != expected:
            raise ValueError(f"Prepared design must have {expected} features, got {prepared.matrix.shape[1]}.")


def _as_2d(X) -> np.ndarray:
    X = np.asarray(X, dtype=float)
    if X.ndim == 1:
        X = X.reshape(1, -1)
    if X.ndim != 2:
        raise ValueError(f"X must have shape (n, d), got {X.shape}.")
    return X


def segment_residuals(x, y, row_offsets, dims, features, beta, *, x_offsets=None, stream=None):
    """Per segment k: (sum (y - phi(x) . beta_k)^2, sum y^2) on the device.

    ``beta`` is (K, stride) with each segment's coefficients in its model's
    feature order; returns two float64 tensors of length K.
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
    if x_offsets is None:
        x_offsets = ro[:-1] * dims_t.to(t.int64)
    xo = to_device(x_offsets, t.int64, dev)
    b = to_device(beta, t.float64, dev)
    sse = t.empty(K, dtype=t.float64, device=dev)
    ssy = t.empty(K, dtype=t.float64, device=dev)
    seg = N.ArtSegments(K, ptr(ro), ptr(xo), ptr(dims_t), ptr(feats))
    N.check(lib.art_segment_residuals(C.byref(seg), ptr(x), ptr(y), ptr(b), int(b.shape[1]), ptr(sse), ptr(ssy),
                                      stream_handle(stream)), "art_segment_residuals")
    sse._keepalive = (x, y, ro, xo, dims_t, feats, b)
    return sse, ssy


def fit_models_batched(template, Xs, ys, *, precision: Precision = "fp64", stream=None) -> list:
    """Unweighted fits of one model template to several datasets in one launch.

    Entry k is ``template.clone().fit(Xs[k], ys[k])`` -- the same trace-scaled
    ridge solve, solver policy and diagnostics as the single-node fit -- or
    the exception that call raises.  All systems go to the device together in
    one ``art_ridge_batched`` call (the mixed form refines its solutions to
    the FP64 form's tolerance), so a tree level costs one launch sequence and
    one read of the results instead of one of each per node.
    """

    if not Xs:
        return []
    if isinstance(template, PolynomialRidgeModel) and template.degree not in (1, 2):
        raise ValueError("batched fits support affine and degree 1/2 polynomial models")
    kind = template.kind() if isinstance(template, PolynomialRidgeModel) else N.FEATURES_AFFINE
    Xs = [_as_2d(X) for X in Xs]
    ys = [np.asarray(y, dtype=float).reshape(-1) for y in ys]
    d = Xs[0].shape[1]
    if any(X.shape[1] != d for X in Xs) or any(X.shape[0] != y.shape[0] for X, y in zip(Xs, ys)):
        raise ValueError("every dataset needs the same dimension and one y per row")
    p = kind_feature_count(d, kind)
    ro = np.concatenate([[0], np.cumsum([X.shape[0] for X in Xs])]).astype(np.int64)
    K = len(Xs)
    out = solve_weighted_ridge_batched(
        np.concatenate([X.reshape(-1) for X in Xs]), np.concatenate(ys), None, ro, [d] * K, [kind] * K,
        [float(template.ridge)] * K, weight_floor=1e-12, solver=template.solver, precision=precision,
        auto_rcond_threshold=template.auto_rcond_threshold, max_features=p, max_dim=d, condition=True,
        stream=stream)
    beta, lam = out.beta.cpu().numpy(), out.ridge_effective.cpu().numpy()
    cond, status, info = out.cond_estimate.cpu().numpy(), out.status.cpu().numpy(), out.info.cpu().numpy()
    models = []
    for k in range(K):
        st = int(status[k])
        if st > 0:
            models.append(np.linalg.LinAlgError(
                "Normal-equation Cholesky factorization failed; use solver='auto', "
                "solver='qr', or solver='svd', or increase ridge regularization."))
            continue
        if st in (-1, -2):
            models.append(ValueError("design, y and weights must be finite and weights nonnegative."))
            continue
        if st == -3:
            models.append(np.linalg.LinAlgError("Ridge solve produced non-finite coefficients."))
            continue
        if st < 0:
            models.append(RuntimeError(f"art_ridge_batched status {st}"))
            continue
        m = template.clone()
        m.solve_result_ = _result_from_row(beta[k], lam[k], cond[k], st, int(info[k]), p, template.solver)
        m.coef_ = m.solve_result_.coefficients
        if isinstance(m, PolynomialRidgeModel):
            m._set_transformer(d)
        models.append(m)
    return models
