"""Coarse build and splitter timing (reference art/timing.py:21-131), plus device timing.

``BuildTimingProfile`` and ``SplitterTimingProfile`` keep the reference's
field names; ``DeviceTimer`` brackets stream work with CUDA events and reads
them lazily, so timing never adds a host synchronisation inside a build.
"""

from __future__ import annotations

from contextlib import contextmanager
from dataclasses import dataclass, field
from time import perf_counter
from typing import Iterator, Literal

BuildTimingCategory = Literal["sampling", "splitter", "model_refit"]
SplitterTimingCategory = Literal["least_squares", "backtracking", "gradient", "sigmoid"]


@dataclass
class BuildTimingProfile:
    sampling_seconds: float = 0.0
    splitter_seconds: float = 0.0
    optimizer_model_refit_seconds: float = 0.0

    @contextmanager
    def measure(self, category: BuildTimingCategory) -> Iterator[None]:
        start = perf_counter()
        try:
            yield
        finally:
            dt = perf_counter() - start
            if category == "sampling":
                self.sampling_seconds += dt
            elif category == "splitter":
                self.splitter_seconds += dt
            else:
                self.optimizer_model_refit_seconds += dt

    def summary(self, total_build_seconds: float) -> dict[str, float]:
        total = max(float(total_build_seconds), 0.0)
        other = max(total - self.sampling_seconds - self.splitter_seconds, 0.0)

        def pct(v):
            return 0.0 if total == 0.0 else 100.0 * v / total

        return {
            "total_build_seconds": total,
            "sampling_seconds": self.sampling_seconds, "sampling_percent": pct(self.sampling_seconds),
            "splitter_seconds": self.splitter_seconds, "splitter_percent": pct(self.splitter_seconds),
            "optimizer_model_refit_seconds": self.optimizer_model_refit_seconds,
            "optimizer_model_refit_percent": pct(self.optimizer_model_refit_seconds),
            "other_seconds": other, "other_percent": pct(other),
        }


@dataclass
class SplitterTimingProfile:
    least_squares_seconds: float = 0.0
    backtracking_seconds: float = 0.0
    gradient_seconds: float = 0.0
    sigmoid_seconds: float = 0.0
    least_squares_count: int = 0
    backtracking_count: int = 0
    gradient_count: int = 0
    sigmoid_count: int = 0
    line_search_candidate_count: int = 0

    @contextmanager
    def measure(self, category: SplitterTimingCategory, *, count: bool = False) -> Iterator[None]:
        start = perf_counter()
        try:
            yield
        finally:
            setattr(self, f"{category}_seconds", getattr(self, f"{category}_seconds") + perf_counter() - start)
            if count:
                setattr(self, f"{category}_count", getattr(self, f"{category}_count") + 1)

    def count_line_search_candidate(self) -> None:
        self.line_search_candidate_count += 1

    def summary(self, total_seconds: float) -> dict[str, float | int]:
        total = max(float(total_seconds), 0.0)
        phases = {k: getattr(self, k) for k in ("least_squares_seconds", "backtracking_seconds",
                                                   "gradient_seconds", "sigmoid_seconds")}
        out: dict[str, float | int] = {"total_seconds": total, **phases}
        for k in ("least_squares_count", "backtracking_count", "gradient_count", "sigmoid_count",
                  "line_search_candidate_count"):
            out[k] = getattr(self, k)
        for k, v in phases.items():
            out[k.replace("_seconds", "_percent")] = 0.0 if total == 0.0 else 100.0 * v / total
        return out


@dataclass
class DeviceTimer:
    """Accumulates device time of bracketed stream work per category (CUDA events)."""

    pending: list = field(default_factory=list)
    totals_ms: dict = field(default_factory=dict)

    @contextmanager
    def measure(self, category: str, stream=None) -> Iterator[None]:
        import torch

        s = torch.cuda.current_stream() if stream is None else stream
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        try:
            yield
        finally:
            b.record(s)
            self.pending.append((category, a, b))

    def summary(self) -> dict[str, float]:
        for cat, a, b in self.pending:
            b.synchronize()
            self.totals_ms[cat] = self.totals_ms.get(cat, 0.0) + a.elapsed_time(b)
        self.pending.clear()
        return dict(self.totals_ms)
