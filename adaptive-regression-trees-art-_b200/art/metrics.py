"""Error metrics for model and tree evaluation (reference art/metrics.py:23-93)."""

from __future__ import annotations

import numpy as np


def _pair(y_true, y_pred):
    a = np.asarray(y_true, dtype=float).reshape(-1)
    b = np.asarray(y_pred, dtype=float).reshape(-1)
    if a.shape != b.shape:
        raise ValueError(f"y_true and y_pred must match, got {a.shape} and {b.shape}.")
    return a, b


def sum_squared_error(y_true, y_pred) -> float:
    a, b = _pair(y_true, y_pred)
    r = a - b
    return float(np.dot(r, r))


def mean_squared_error(y_true, y_pred) -> float:
    a, b = _pair(y_true, y_pred)
    if a.size == 0:
        raise ValueError("Cannot compute mean squared error on an empty array.")
    return sum_squared_error(a, b) / a.size


def relative_l2_error(y_true, y_pred, floor: float = 1e-12) -> float:
    a, b = _pair(y_true, y_pred)
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(a)), float(floor)))


def pointwise_relative_error(y_true, y_pred, floor: float = 1e-12) -> np.ndarray:
    a, b = _pair(y_true, y_pred)
    return np.abs(a - b) / np.maximum(np.abs(a), float(floor))


def pointwise_relative_error_quantile(y_true, y_pred, quantile, floor: float = 1e-12):
    q = np.asarray(quantile, dtype=float)
    if not np.all(np.isfinite(q)) or np.any((q < 0.0) | (q > 1.0)):
        raise ValueError("quantile must contain finite values in [0, 1].")
    out = np.quantile(pointwise_relative_error(y_true, y_pred, floor=floor), q)
    return float(out) if np.ndim(out) == 0 else out


def median_pointwise_relative_error(y_true, y_pred, floor: float = 1e-12) -> float:
    return float(pointwise_relative_error_quantile(y_true, y_pred, 0.5, floor=floor))


def max_pointwise_relative_error(y_true, y_pred, floor: float = 1e-12) -> float:
    return float(np.max(pointwise_relative_error(y_true, y_pred, floor=floor)))
