"""Polytope regions A x <= b and box domains (reference art/domain.py:11-119)."""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass(frozen=True)
class PolytopeRegion:
    """A convex polytope represented by linear inequalities A x <= b."""

    A: np.ndarray
    b: np.ndarray
    depth: int = 0
    tag: Optional[str] = None

    def __post_init__(self) -> None:
        A = np.asarray(self.A, dtype=float)
        b = np.asarray(self.b, dtype=float).reshape(-1)
        if A.ndim != 2:
            raise ValueError(f"A must have shape (m, d), got {A.shape}.")
        if A.shape[0] != b.shape[0]:
            raise ValueError(f"A and b must have compatible rows, got {A.shape[0]} and {b.shape[0]}.")
        object.__setattr__(self, "A", A)
        object.__setattr__(self, "b", b)

    @property
    def dimension(self) -> int:
        return int(self.A.shape[1])

    def contains(self, X: np.ndarray, tol: float = 1e-10) -> np.ndarray:
        """Boolean mask of points satisfying A x <= b + tol (domain.py:40-48)."""

        X = np.asarray(X, dtype=float)
        if X.ndim == 1:
            X = X.reshape(1, -1)
        if X.ndim != 2 or X.shape[1] != self.dimension:
            raise ValueError(f"X must have shape (n, {self.dimension}), got {X.shape}.")
        return np.all(X @ self.A.T <= self.b[None, :] + tol, axis=1)


@dataclass(frozen=True)
class BoxDomain:
    """Axis-aligned box domain with bounds shaped (d, 2)."""

    bounds: np.ndarray

    def __post_init__(self) -> None:
        bounds = np.asarray(self.bounds, dtype=float)
        if bounds.ndim != 2 or bounds.shape[1] != 2:
            raise ValueError(f"bounds must have shape (d, 2), got {bounds.shape}.")
        if np.any(bounds[:, 0] >= bounds[:, 1]):
            raise ValueError("Each bound must satisfy low < high.")
        object.__setattr__(self, "bounds", bounds)

    @property
    def dimension(self) -> int:
        return int(self.bounds.shape[0])

    @classmethod
    def hypercube(cls, dimension: int, low: float, high: float) -> "BoxDomain":
        dimension = int(dimension)
        if dimension < 1:
            raise ValueError("dimension must be at least 1.")
        return cls(np.tile(np.array([[float(low), float(high)]]), (dimension, 1)))

    def as_region(self, depth: int = 0, tag: Optional[str] = "root") -> PolytopeRegion:
        """[I; -I] x <= [highs; -lows] (domain.py:87-92)."""

        d = self.dimension
        A = np.vstack([np.eye(d), -np.eye(d)])
        b = np.concatenate([self.bounds[:, 1], -self.bounds[:, 0]])
        return PolytopeRegion(A=A, b=b, depth=depth, tag=tag)


def split_region(region: PolytopeRegion, w: np.ndarray, z: float, depth: Optional[int] = None,
                 left_tag: Optional[str] = None, right_tag: Optional[str] = None):
    """Left gets w.x <= z, right gets -w.x <= -z (domain.py:95-119)."""

    w = np.asarray(w, dtype=float).reshape(-1)
    if w.shape[0] != region.dimension:
        raise ValueError(f"w must have shape ({region.dimension},), got {w.shape}.")
    child_depth = region.depth + 1 if depth is None else int(depth)
    left = PolytopeRegion(np.vstack([region.A, w[None, :]]), np.concatenate([region.b, [float(z)]]),
                          depth=child_depth, tag=left_tag)
    right = PolytopeRegion(np.vstack([region.A, -w[None, :]]), np.concatenate([region.b, [-float(z)]]),
                           depth=child_depth, tag=right_tag)
    return left, right
