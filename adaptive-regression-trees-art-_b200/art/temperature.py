"""Node-local temperature scales for the soft splitter (reference art/temperature.py:19-164).

T = c * median nearest-neighbour distance of (at most ``max_points``
subsampled) node samples, or c * median pairwise distance * n^(-1/d).
``nn_method="device"`` computes the nearest-neighbour distances and their
median on the GPU (``art_median_nn_distance``, exact brute force in FP64), and
``median_nn_distance_batched`` does it for many point sets in one launch.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass
from typing import Literal

import numpy as np

TemperatureMode = Literal["median_nn", "median_pairwise_scaled"]
NearestNeighborMethod = Literal["kdtree", "bruteforce", "device"]
TemperatureStrategy = Literal["splitter", "fixed", "tune_root", "tune_node"]
DEFAULT_TEMPERATURE_GRID = (1e-4, 5e-4, 0.001, 0.005, 0.01, 0.05, 0.1, 0.5, 1.0)


@dataclass(frozen=True)
class TemperatureConfig:
    strategy: TemperatureStrategy = "fixed"
    scale_mode: TemperatureMode = "median_nn"
    c: float = 0.1
    c_values: tuple[float, ...] = DEFAULT_TEMPERATURE_GRID
    validation_fraction: float = 0.2
    max_points: int | None = 512
    nn_method: NearestNeighborMethod | None = None
    bruteforce_dimension_threshold: int = 20

    def __post_init__(self) -> None:
        if self.strategy not in ("splitter", "fixed", "tune_root", "tune_node"):
            raise ValueError("Unknown temperature strategy.")
        if self.c <= 0.0:
            raise ValueError("Temperature c must be positive.")
        if not self.c_values or any(v <= 0.0 for v in self.c_values):
            raise ValueError("Temperature c_values must be nonempty and positive.")
        if not (0.0 < self.validation_fraction < 0.5):
            raise ValueError("validation_fraction must satisfy 0 < fraction < 0.5.")
        if self.max_points is not None and self.max_points < 2:
            raise ValueError("max_points must be at least 2 or None.")
        if self.bruteforce_dimension_threshold < 1:
            raise ValueError("bruteforce_dimension_threshold must be at least 1.")


def subsample_points(X, max_points: int | None = 512, random_state=None) -> np.ndarray:
    X = np.asarray(X, dtype=float)
    if X.ndim != 2:
        raise ValueError(f"X must have shape (n, d), got {X.shape}.")
    if max_points is None or X.shape[0] <= max_points:
        return X
    if max_points < 1:
        raise ValueError("max_points must be positive or None.")
    rng = random_state if isinstance(random_state, np.random.Generator) else np.random.default_rng(random_state)
    return X[rng.choice(X.shape[0], size=int(max_points), replace=False)]


def pairwise_distances(X) -> np.ndarray:
    X = np.asarray(X, dtype=float)
    if X.ndim != 2:
        raise ValueError(f"X must have shape (n, d), got {X.shape}.")
    return np.linalg.norm(X[:, None, :] - X[None, :, :], axis=2)


def median_nearest_neighbor_distance(X, method: NearestNeighborMethod = "kdtree") -> float:
    X = np.asarray(X, dtype=float)
    if X.ndim != 2:
        raise ValueError(f"X must have shape (n, d), got {X.shape}.")
    if X.shape[0] < 2:
        raise ValueError("At least two points are required.")
    if method not in ("kdtree", "bruteforce", "device"):
        raise ValueError("method must be 'kdtree', 'bruteforce' or 'device'.")
    if method == "device":
        return float(median_nn_distance_batched([X])[0].item())
    if method == "kdtree":
        try:
            from scipy.spatial import cKDTree
        except ImportError:
            warnings.warn("scipy.spatial.cKDTree is unavailable; using brute force.", RuntimeWarning, stacklevel=2)
        else:
            dist, _ = cKDTree(X).query(X, k=2)
            return float(np.median(dist[:, 1]))
    D = pairwise_distances(X)
    np.fill_diagonal(D, np.inf)
    return float(np.median(np.min(D, axis=1)))


def median_nn_distance_batched(point_sets, c: float = 1.0, stream=None):
    """c * median nearest-neighbour distance of each point set, on the GPU.

    ``point_sets`` is a list of (m_k, d_k) arrays (numpy or torch), each at
    most ``MEDIAN_NN_MAX_SET`` points.  Returns a float64 CUDA tensor of K
    values, NaN for sets of fewer than two points.  Distances are exact FP64
    brute force, so they equal the kd-tree query's up to the summation order
    of the squared coordinates.
    """

    from . import _native as N
    from ._device import ptr, require_cuda, stream_handle, to_device, torch

    t = torch()
    dev = require_cuda()
    lib = N.load_library()
    if not (c > 0.0):
        raise ValueError("c must be positive.")
    sets = [np.asarray(P.cpu() if isinstance(P, t.Tensor) else P, dtype=float) for P in point_sets]
    K = len(sets)
    for P in sets:
        if P.ndim != 2:
            raise ValueError(f"X must have shape (n, d), got {P.shape}.")
    sizes = np.array([P.shape[0] for P in sets], dtype=np.int64)
    if K and sizes.max() > N.MEDIAN_NN_MAX_SET:
        raise ValueError(f"at most {N.MEDIAN_NN_MAX_SET} points per set are supported")
    out = t.empty(K, dtype=t.float64, device=dev)
    if K == 0:
        return out
    dims = np.array([P.shape[1] for P in sets], dtype=np.int32)
    x_off = np.concatenate([[0], np.cumsum(sizes * dims)[:-1]]).astype(np.int64)
    s_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    rows = np.concatenate([np.arange(m, dtype=np.int64) for m in sizes]) if sizes.sum() else np.zeros(1, np.int64)
    xd = to_device(np.concatenate([P.reshape(-1) for P in sets]) if sizes.sum() else np.zeros(1), t.float64, dev)
    xo, dd, so, rr = (to_device(a, None, dev) for a in (x_off, dims, s_off, rows))
    rc = lib.art_median_nn_distance(K, ptr(xd), ptr(xo), ptr(dd), ptr(so), ptr(rr), int(sizes.max()), float(c),
                                    ptr(out), stream_handle(stream))
    N.check(rc, "art_median_nn_distance")
    out._keepalive = (xd, xo, dd, so, rr)
    return out


def median_pairwise_distance(X) -> float:
    X = np.asarray(X, dtype=float)
    if X.shape[0] < 2:
        raise ValueError("At least two points are required.")
    D = pairwise_distances(X)
    return float(np.median(D[np.triu_indices(X.shape[0], k=1)]))


def estimate_temperature(X, mode: TemperatureMode, c: float = 1.0, max_points: int | None = 512,
                         random_state=None, nn_method: NearestNeighborMethod = "kdtree") -> float:
    used = subsample_points(X, max_points=max_points, random_state=random_state)
    if c <= 0.0:
        raise ValueError("c must be positive.")
    if mode == "median_nn":
        base = median_nearest_neighbor_distance(used, method=nn_method)
    elif mode == "median_pairwise_scaled":
        base = median_pairwise_distance(used) * used.shape[0] ** (-1.0 / used.shape[1])
    else:
        raise ValueError("mode must be 'median_nn' or 'median_pairwise_scaled'.")
    T = float(c) * float(base)
    if not np.isfinite(T) or T <= 0.0:
        raise RuntimeError("Estimated temperature is not positive and finite.")
    return T


def temperature_grid(X, mode: TemperatureMode, c_values, max_points: int | None = 512, random_state=None,
                     nn_method: NearestNeighborMethod = "kdtree") -> list[float]:
    temps = [estimate_temperature(X, mode=mode, c=float(c), max_points=max_points, random_state=random_state,
                                  nn_method=nn_method) for c in c_values]
    unique: list[float] = []
    for T in temps:
        if not any(np.isclose(T, u) for u in unique):
            unique.append(T)
    return unique
