"""Step-size control and Armijo backtracking (reference art/optimizers.py:11-121).

These host objects keep the reference's API for callers that drive a line
search themselves; the split search runs the same rules on the device
(``art_split_level``).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np


@dataclass
class LineSearchResult:
    theta: np.ndarray
    value: float
    step_size: float
    success: bool
    n_backtracks: int


@dataclass
class AdaptiveAlpha:
    """Next initial step: x grow after an immediate success, x recovery after a
    heavy search, / rho after a moderate one, the failed step x rho after a
    failure; always clipped to [alpha_min, alpha_max]."""

    alpha: float = 1.0
    alpha_min: float = 1e-12
    alpha_max: float = 1e3
    grow: float = 10.0
    recovery: float = 10.0
    heavy_backtrack_threshold: int = 8

    def __post_init__(self) -> None:
        if self.alpha <= 0.0 or self.alpha_min <= 0.0:
            raise ValueError("alpha and alpha_min must be positive.")
        if self.alpha_max < self.alpha_min:
            raise ValueError("alpha_max must be at least alpha_min.")
        if self.grow < 1.0 or self.recovery < 1.0:
            raise ValueError("grow and recovery must be at least 1.")
        if self.heavy_backtrack_threshold < 0:
            raise ValueError("heavy_backtrack_threshold must be nonnegative.")
        self.alpha = self._clip(self.alpha)

    def update(self, result: LineSearchResult, rho: float) -> float:
        if not (0.0 < rho < 1.0):
            raise ValueError("rho must satisfy 0 < rho < 1.")
        if not result.success:
            self.alpha = self._clip(result.step_size * rho)
        elif result.n_backtracks == 0:
            self.alpha = self._clip(result.step_size * self.grow)
        elif result.n_backtracks >= self.heavy_backtrack_threshold:
            self.alpha = self._clip(result.step_size * self.recovery)
        else:
            self.alpha = self._clip(result.step_size / rho)
        return self.alpha

    def _clip(self, alpha: float) -> float:
        return min(max(float(alpha), self.alpha_min), self.alpha_max)


def armijo_backtracking(value_fn: Callable[[np.ndarray], float], candidate_fn: Callable[[float], np.ndarray],
                        current_value: float, directional_derivative: float, alpha0: float = 1.0,
                        rho: float = 0.5, c: float = 1e-4, max_backtracks: int = 25) -> LineSearchResult:
    """First alpha0 * rho^k (k <= max_backtracks) with f <= f0 + c alpha slope."""

    if alpha0 <= 0.0:
        raise ValueError("alpha0 must be positive.")
    if not (0.0 < rho < 1.0) or not (0.0 < c < 1.0):
        raise ValueError("rho and c must lie strictly between 0 and 1.")
    if max_backtracks < 0:
        raise ValueError("max_backtracks must be nonnegative.")
    if directional_derivative >= 0.0:
        raise ValueError("directional_derivative must be negative for a descent direction.")
    alpha = float(alpha0)
    theta = candidate_fn(alpha)
    value = float(value_fn(theta))
    for k in range(max_backtracks + 1):
        if k > 0:
            alpha *= rho
            theta = candidate_fn(alpha)
            value = float(value_fn(theta))
        if value <= current_value + c * alpha * directional_derivative:
            return LineSearchResult(np.asarray(theta, float), value, alpha, True, k)
    return LineSearchResult(np.asarray(theta, float), value, alpha, False, max_backtracks)
