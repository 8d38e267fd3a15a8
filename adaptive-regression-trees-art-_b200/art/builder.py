"""Adaptive regression-tree builder (drop-in for the reference art/builder.py).

The node policy is the reference's (builder.py:116-1251): children are topped
up to the target sample count by hit-and-run inside their polytope, a ridge
model is fitted, tolerance and depth stop the recursion, otherwise a soft
oblique split is searched, retried, checked and turned into two child
polytopes whose inherited samples follow ``(X @ w - z) >= 0 -> right``.
Every numeric step runs on the GPU kernels: node fits (``art_ridge_batched``),
split searches (``art_split_level``) and hit-and-run top-ups
(``art_hit_and_run``).  With ``traversal="bfs"`` and the default
``level_dispatch=True`` a whole ready cohort is split in one launch sequence
(the reference's BatchedSplitDispatcher role, _cuda_batched_builder.py:18-101),
replayed from a captured CUDA graph per level shape class when
``cuda_graphs=True`` (the default; see ``art.graphs``).

Random streams are consumed in the reference's order (seeds from
``_next_seed``, host draws for sampler directions and splitter
initialisation), so a build with the same ``random_state`` reproduces the
reference's tree decisions; with ``traversal="bfs"`` this holds while no
split retry happens (retries draw their seeds after the cohort's first
attempts, as the reference's batched dispatcher does).
"""

from __future__ import annotations

import copy
from contextlib import nullcontext
from dataclasses import dataclass, field, replace
from time import perf_counter
from typing import Callable, Iterator, Literal

import numpy as np

from .domain import BoxDomain, PolytopeRegion, split_region
from .metrics import mean_squared_error, relative_l2_error
from .models import (
    AffineRidgeModel,
    MODEL_CONDITION_WARNING_THRESHOLD,
    PolynomialRidgeModel,
    PreparedDesign,
    PreparedFeatureModel,
    RegressionModel,
    WeightedRegressionModel,
    model_effective_dimension,
    ridge_solve_diagnostics,
)
from .sampling import (
    HitAndRunSampler,
    Sampler,
    covariance_eigendecomposition_batched,
    floor_covariance_eigenvalues,
    sample_covariance_eigendecomposition,
    sample_uniform_box,
)
from .splitters import SoftObliqueSplitter, SplitNotFoundError, SplitResult, Splitter
from .temperature import TemperatureConfig, estimate_temperature
from .timing import BuildTimingCategory, BuildTimingProfile
from .tree import LeafNode, RegressionTree, SplitNode, TreeNode

ErrorMetric = Callable[[np.ndarray, np.ndarray], float]
SampleCountPolicy = Callable[[RegressionModel, int], int]


@dataclass(frozen=True)
class TreeBuildResult:
    tree: RegressionTree
    oracle_queries: int
    restarts_on_failure: int
    build_timing: dict[str, float] | None = None


@dataclass
class _NodeSamples:
    X: np.ndarray
    y: np.ndarray
    n_inherited: int
    n_new: int
    sampling_metadata: dict[str, object] = field(default_factory=dict)


@dataclass(slots=True)
class _NodeWork:
    """One node from inherited samples to a prepared split candidate."""

    region: PolytopeRegion
    samples: _NodeSamples
    depth: int
    node_id: str
    parent: SplitNode | None = None
    side: Literal["left", "right"] | None = None
    model: RegressionModel | None = None
    parent_mse: float = 0.0
    metadata: dict[str, object] = field(default_factory=dict)
    convergence: dict[str, object] = field(default_factory=dict)
    prepared: PreparedDesign | None = None
    topped: bool = False                      # samples already topped up (cohort launch)
    topup_error: Exception | None = None      # the top-up's failure, raised at prepare
    topup_pending: tuple | None = None        # cohort top-up awaiting its oracle values
    fit_cache: tuple | None = None            # (model, predictions) or (exception, None) from a cohort fit


@dataclass
class _SplitState:
    """Temperature and retry bookkeeping shared by scalar and cohort dispatch."""

    temperature: float | None
    context: dict[str, object]
    limit: int
    min_side_fallback: bool
    retries: int = 0
    reasons: list[str] = field(default_factory=list)

    @property
    def fallback(self) -> bool:
        return self.min_side_fallback and self.retries >= self.limit

    @property
    def metadata(self) -> dict[str, object]:
        return {"restarts_on_failure": self.retries, "split_attempt_failure_reasons": tuple(self.reasons)}

    def error(self, exc: SplitNotFoundError) -> SplitNotFoundError:
        return SplitNotFoundError(exc.reason, str(exc), diagnostics=exc.diagnostics,
                                  restarts_on_failure=self.retries, failure_reasons=tuple(self.reasons),
                                  context=self.context)


@dataclass
class RegressionTreeBuilder:
    """Build a regression tree by DFS (default) or FIFO level cohorts (BFS) on the GPU."""

    domain: BoxDomain | PolytopeRegion
    oracle: Callable[[np.ndarray], float | np.ndarray]
    model_template: RegressionModel
    splitter: Splitter
    error_threshold: float
    max_depth: int = 10
    error_metric: ErrorMetric = relative_l2_error
    sample_multiplier: int = 50
    sample_count: int | SampleCountPolicy | None = None
    sampler: Sampler = field(default_factory=lambda: HitAndRunSampler(burn_in=0, thinning=20))
    root_sampler: Sampler = field(default_factory=HitAndRunSampler)
    exact_box_root: bool = True
    isotropic_sampling: bool = True
    isotropic_pilot_multiplier: int = 50
    temperature_config: TemperatureConfig | None = None
    min_split_gain: float = 0.0
    min_relative_split_gain: float = 0.0
    max_retries_on_failure: int = 0
    validation_fraction: float = 0.0
    store_samples: bool = False
    store_leaf_representative: bool = False
    store_diagnostics: bool = False
    profile_build_timing: bool = False
    oracle_vectorized: bool = False
    random_state: int | np.random.Generator | None = None
    traversal: Literal["dfs", "bfs"] = "dfs"
    node_batch_size: int = 20
    batch_reorder: bool = True
    check_split_gain: bool = False
    level_dispatch: bool = True
    cuda_graphs: bool = True
    cohort_top_up: bool = True
    batched_temperature_tuning: bool = True
    batched_fits: bool = True
    fit_precision: Literal["fp64", "mixed"] = "fp64"
    refinement_rounds: int = 0
    refinement_points: int = 1024
    refinement_leaves: int = 4
    verbose: bool = False

    oracle_queries: int = field(default=0, init=False)
    restarts_on_failure: int = field(default=0, init=False)
    _rng: np.random.Generator = field(init=False, repr=False)
    _root_temperature_c: float | None = field(default=None, init=False, repr=False)
    _target_samples: int = field(init=False, repr=False)
    _effective_dimension: int | None = field(init=False, repr=False)
    _timing_profile: BuildTimingProfile | None = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        if self.traversal not in ("dfs", "bfs"):
            raise ValueError("traversal must be 'dfs' or 'bfs'.")
        if (not isinstance(self.node_batch_size, (int, np.integer)) or isinstance(self.node_batch_size, (bool, np.bool_))
                or self.node_batch_size < 1):
            raise ValueError("node_batch_size must be a positive integer.")
        self.node_batch_size = int(self.node_batch_size)
        if not isinstance(self.batch_reorder, (bool, np.bool_)):
            raise ValueError("batch_reorder must be a boolean.")
        if not isinstance(self.check_split_gain, (bool, np.bool_)):
            raise ValueError("check_split_gain must be a boolean.")
        if self.error_threshold < 0.0:
            raise ValueError("error_threshold must be nonnegative.")
        if self.max_depth < 0:
            raise ValueError("max_depth must be nonnegative.")
        if self.sample_multiplier < 1:
            raise ValueError("sample_multiplier must be at least 1.")
        if self.min_split_gain < 0.0 or self.min_relative_split_gain < 0.0:
            raise ValueError("Split-gain thresholds must be nonnegative.")
        if self.max_retries_on_failure < 0:
            raise ValueError("max_retries_on_failure must be nonnegative.")
        if not (0.0 <= self.validation_fraction < 1.0):
            raise ValueError("validation_fraction must satisfy 0 <= fraction < 1.")
        if self.isotropic_sampling and self.isotropic_pilot_multiplier < 2:
            raise ValueError("isotropic_pilot_multiplier must be at least 2.")
        if self.isotropic_sampling and not isinstance(self.sampler, HitAndRunSampler):
            raise TypeError("isotropic_sampling requires a HitAndRunSampler.")
        root_hr = not (isinstance(self.domain, BoxDomain) and self.exact_box_root)
        if self.isotropic_sampling and root_hr and not isinstance(self.root_sampler, HitAndRunSampler):
            raise TypeError("isotropic_sampling requires a HitAndRunSampler for non-exact roots.")
        if self.max_retries_on_failure > 0 and int(getattr(self.splitter, "n_restarts", 1)) != 1:
            raise ValueError("max_retries_on_failure requires splitter.n_restarts == 1.")
        if not isinstance(self.splitter, SoftObliqueSplitter):
            raise TypeError("the B200 builder drives the GPU SoftObliqueSplitter")
        self._rng = (self.random_state if isinstance(self.random_state, np.random.Generator)
                     else np.random.default_rng(self.random_state))
        self._effective_dimension = self._resolve_effective_dimension()
        self._target_samples = self._resolve_sample_count()
        if self._target_samples < 2:
            raise ValueError("The node sample count must be at least 2.")
        if not isinstance(self.model_template, WeightedRegressionModel):
            raise TypeError("SoftObliqueSplitter requires a model with fit_weighted support.")
        if self.validation_fraction > 0.0 and self._metric_name() != "max_pointwise_relative_error":
            raise ValueError("validation_fraction requires max_pointwise_relative_error.")
        if self.fit_precision not in ("fp64", "mixed"):
            raise ValueError("fit_precision must be 'fp64' or 'mixed'.")
        if self.refinement_rounds < 0 or self.refinement_points < 1 or self.refinement_leaves < 1:
            raise ValueError("refinement needs rounds >= 0, points >= 1 and leaves >= 1.")
        if self.temperature_config is None:
            self.temperature_config = TemperatureConfig()
        if (self.temperature_config.strategy in ("tune_root", "tune_node") and self._target_samples < 4):
            raise ValueError("Temperature tuning requires at least four node samples.")
        if self.hard_refits and self.verbose:
            print("Final hard refits enabled.")

    # ---------------------------------------------------------------- public
    @property
    def hard_refits(self) -> bool:
        """Hard losses are needed for gain checks, restart selection or tuning (builder.py:264-269)."""
        return (self.check_split_gain or self.splitter.n_restarts != 1
                or self.temperature_config.strategy not in ("fixed", "splitter"))

    @property
    def dimension(self) -> int:
        return self.domain.dimension

    @property
    def target_samples(self) -> int:
        return self._target_samples

    def build(self) -> TreeBuildResult:
        """Build a fresh tree and reset all per-build state (builder.py:279-345)."""

        self._timing_profile = BuildTimingProfile() if self.profile_build_timing else None
        start = perf_counter() if self._timing_profile is not None else None
        self.oracle_queries = 0
        self.restarts_on_failure = 0
        self._root_temperature_c = None
        root_region = self.domain.as_region() if isinstance(self.domain, BoxDomain) else self.domain
        X_root, meta = self._sample_root(root_region)
        y_root = self._query_oracle(X_root)
        work = _NodeWork(root_region, _NodeSamples(X_root, y_root, 0, X_root.shape[0], meta), depth=0,
                         node_id="root")
        self._leaf_samples = {} if self.refinement_rounds else None
        root = self._grow(work)
        for _ in range(self.refinement_rounds):
            root = self._refine_round(root)
        tree = RegressionTree(root=root, oracle_queries=self.oracle_queries, metadata={
            "error_metric": self._metric_name(), "error_threshold": self.error_threshold,
            "effective_dimension": self._effective_dimension, "splitter": type(self.splitter).__name__,
            "optimizer": "b200", "check_split_gain": self.check_split_gain, "hard_refits": self.hard_refits,
            "traversal": self.traversal,
            "node_batch_size": self.node_batch_size if self.traversal == "bfs" else 1,
            "target_samples_per_node": self._target_samples, "restarts_on_failure": self.restarts_on_failure,
            "validation_fraction": self.validation_fraction, "isotropic_sampling": self.isotropic_sampling,
            "isotropic_pilot_multiplier": self.isotropic_pilot_multiplier,
            "temperature_strategy": self.temperature_config.strategy,
        })
        timing = None
        if self._timing_profile is not None and start is not None:
            timing = self._timing_profile.summary(perf_counter() - start)
        tree.metadata["build_timing"] = timing
        return TreeBuildResult(tree=tree, oracle_queries=self.oracle_queries,
                               restarts_on_failure=self.restarts_on_failure, build_timing=timing)

    def _grow(self, work: _NodeWork) -> TreeNode:
        if self.traversal == "dfs":
            return self._build_node(work)
        from ._batched_builder import build_bfs

        dispatch = LevelSplitDispatcher(self) if self.level_dispatch else None
        return build_bfs(self, work, dispatch)

    def _refine_round(self, root: TreeNode) -> TreeNode:
        """One adaptive refinement round (the reference has no driver for this).

        The ``refinement_leaves`` leaves with the largest fit error (ties in
        depth-first order) get ``refinement_points`` new samples between them
        (the first ones one more when the count does not divide), drawn by the
        builder's sampler inside each leaf's region from one of its samples
        and queried from the oracle.  Each leaf, in that order, is then
        rebuilt from its samples plus the new ones through the builder's own
        node policy (fit, stopping rules, split, children topped up to the
        target count), and the subtree replaces it.
        """

        tree = RegressionTree(root=root)
        leaves = [n for n in tree.iter_nodes() if isinstance(n, LeafNode)]
        order = sorted(range(len(leaves)), key=lambda i: -float(leaves[i].metadata.get("fit_error", 0.0)))
        chosen = [leaves[i] for i in order[: self.refinement_leaves]]
        base, extra = divmod(self.refinement_points, len(chosen))
        for q, leaf in enumerate(chosen):
            smp = self._leaf_samples[leaf.node_id]
            m = base + (1 if q < extra else 0)
            if m == 0:
                continue
            x0 = smp.X[int(self._rng.integers(0, smp.X.shape[0]))]
            X_new, meta = self._sample_region(leaf.region, m, x0=x0, sampler=self.sampler)
            y_new = self._query_oracle(X_new)
            work = _NodeWork(leaf.region, _NodeSamples(np.vstack([smp.X, X_new]), np.concatenate([smp.y, y_new]),
                                                       smp.X.shape[0], m, meta), depth=leaf.depth, node_id=leaf.node_id)
            sub = self._grow(work)
            path = RegressionTree(root=root).path_to_node(leaf.node_id)
            if len(path) == 1:
                root = sub
            else:
                parent = path[-2]
                setattr(parent, "left" if parent.left is leaf else "right", sub)
        return root

    # ---------------------------------------------------------------- nodes
    def _build_node(self, work: _NodeWork) -> TreeNode:
        leaf = self._prepare_node(work)
        if leaf is not None:
            return leaf
        node = self._split_node(work)
        if isinstance(node, SplitNode):
            for child in self._children(work, node):
                setattr(node, child.side, self._build_node(child))
        return node

    def _prepare_node(self, work: _NodeWork) -> LeafNode | None:
        """Top up a child, fit its model and apply the stopping rules (builder.py:358-400)."""

        if work.parent is not None:
            inherited = work.samples
            try:
                if work.topped:
                    if work.topup_error is not None:
                        raise work.topup_error
                else:
                    work.samples = self._top_up_child(work.region, inherited.X, inherited.y)
            except (RuntimeError, ValueError) as exc:
                prepared = self._prepare_design(inherited.X)
                model, pred = self._fit_node_model(inherited.X, inherited.y, prepared)
                meta = self._node_metadata(inherited, float(self.error_metric(inherited.y, pred)),
                                           mean_squared_error(inherited.y, pred), model)
                meta["sampling_error"] = repr(exc)
                return self._make_leaf(model, work.region, work.depth, work.node_id, "sampling_failed", meta,
                                       inherited)
        samples = work.samples
        work.prepared = self._prepare_design(samples.X)
        if self.validation_fraction > 0.0:
            work.model, pred, n_fit = self._fit_convergence_model(samples.X, samples.y, work.prepared)
            fit_error = float(self.error_metric(samples.y, pred))
            work.parent_mse = mean_squared_error(samples.y, pred)
            work.convergence = {"convergence_error": fit_error, "convergence_fit_samples": n_fit}
            work.metadata = {**self._node_metadata(samples, fit_error, work.parent_mse, work.model),
                             **work.convergence}
        else:
            cached, work.fit_cache = work.fit_cache, None
            work.model, fit_error, work.parent_mse, work.metadata = self._fit_full_node_model(
                samples, work.prepared, cached=cached)
        if fit_error <= self.error_threshold:
            return self._work_leaf(work, "tolerance_met")
        if work.depth >= self.max_depth:
            return self._work_leaf(work, "max_depth")
        return None

    def _split_node(self, work: _NodeWork) -> TreeNode:
        try:
            result, temperature, retry = self._fit_split(work.samples.X, work.samples.y, work.model,
                                                         work.parent_mse, work.depth, work.prepared)
        except SplitNotFoundError as exc:
            return self._finish_node(work, exc)
        return self._finish_node(work, result, {**temperature, **retry})

    def _finish_node(self, work: _NodeWork, result, context=None) -> TreeNode:
        """Leaf or provisional split node for a final split outcome (builder.py:413-448)."""

        if isinstance(result, SplitNotFoundError):
            return self._work_leaf(work, result.reason, error=result)
        rejection = self._split_rejection_reason(result)
        if rejection is not None:
            return self._work_leaf(work, rejection, result=result, context=context)
        regions = split_region(work.region, result.w, result.z, depth=work.depth + 1,
                               left_tag=f"{work.node_id}/L", right_tag=f"{work.node_id}/R")
        left = LeafNode(result.left_model if result.has_hard_fit else work.model, regions[0], work.depth + 1,
                        f"{work.node_id}/L", status="pending")
        right = LeafNode(result.right_model if result.has_hard_fit else work.model, regions[1], work.depth + 1,
                         f"{work.node_id}/R", status="pending")
        meta = self._split_metadata(work, result, context)
        self._store_samples(meta, work.samples)
        work.prepared = None
        return SplitNode(w=result.w, z=result.z, left=left, right=right, region=work.region, depth=work.depth,
                         node_id=work.node_id, status="split_with_warnings" if meta["warnings"] else "split",
                         metadata=meta)

    def _split_metadata(self, work, result, context):
        meta = {**work.metadata, **self._split_summary(result), **(context or {}),
                "warnings": self._combine_warnings(work.metadata.get("warnings", ()), self._split_warnings(result))}
        if self.store_diagnostics:
            meta["splitter_metadata"] = copy.deepcopy(result.metadata)
        return meta

    def _work_leaf(self, work, status, *, result=None, error=None, context=None):
        if self.validation_fraction > 0.0:
            work.model, _, _, work.metadata = self._fit_full_node_model(work.samples, work.prepared,
                                                                        extra_metadata=work.convergence)
        if error is not None:
            meta = {**work.metadata, **error.context, "split_failure_reason": error.reason,
                    "restarts_on_failure": error.restarts_on_failure,
                    "split_attempt_failure_reasons": error.failure_reasons,
                    "warnings": self._combine_warnings(work.metadata.get("warnings", ()),
                                                       self._diagnostic_warnings(error.diagnostics))}
            if self.store_diagnostics and error.diagnostics is not None:
                meta["splitter_metadata"] = copy.deepcopy(error.diagnostics)
        elif result is not None:
            meta = self._split_metadata(work, result, context)
        else:
            meta = work.metadata
        work.prepared = None
        return self._make_leaf(work.model, work.region, work.depth, work.node_id, status, meta, work.samples)

    def _children(self, work: _NodeWork, node: SplitNode) -> Iterator[_NodeWork]:
        """Inherited-only child jobs, left then right (builder.py:487-500)."""

        samples = work.samples
        right = (samples.X @ node.w - node.z) >= 0.0
        for side, mask in (("left", ~right), ("right", right)):
            child = getattr(node, side)
            X, y = samples.X[mask], samples.y[mask]
            yield _NodeWork(child.region, _NodeSamples(X, y, n_inherited=len(X), n_new=0), child.depth,
                            child.node_id, parent=node, side=side)

    def _top_up_cohort(self, jobs) -> None:
        """Top up a cohort's children with one hit-and-run launch.

        Only for the plain sampler with device draws: every child's builder
        draws (subsample, start point, sampler seed) are taken in cohort order
        exactly as the one-child-at-a-time top-up takes them, and each child's
        chain uses its own seed, so the samples are the ones the sequential
        top-ups produce.  Children whose chain reports a failure are redone by
        the sequential path (which reproduces the failure at the same step).
        """

        from .sampling import HitAndRunSampler

        sp = self.sampler
        if (not self.cohort_top_up or type(sp) is not HitAndRunSampler or getattr(sp, "rng_mode", "reference") != "device"
                or sp.direction_eigenvectors is not None or sp.direction_eigenvalues is not None):
            return
        todo = [j for j in jobs if j.parent is not None and not j.topped]
        if len(todo) < 2:
            return
        # a covariance-shaped top-up whose pilot chain fails draws one seed
        # less one child at a time; then the cohort is undone and left to it
        rng_state = copy.deepcopy(self._rng.bit_generator.state)
        queries0 = self.oracle_queries
        saved = [(j, j.samples) for j in todo]
        reqs = []
        with self._timing_context("sampling"):
            for job in todo:
                job.topped = True
                X = np.asarray(job.samples.X, dtype=float)
                y = np.asarray(job.samples.y, dtype=float).reshape(-1)
                if X.shape[0] == 0:
                    job.topup_error = RuntimeError("Cannot seed child sampling without an inherited point.")
                    continue
                if X.shape[0] > self._target_samples:
                    keep = self._rng.choice(X.shape[0], size=self._target_samples, replace=False)
                    X, y = X[keep], y[keep]
                n_inh = X.shape[0]
                n_new = self._target_samples - n_inh
                if n_new == 0:
                    job.samples = _NodeSamples(X, y, n_inh, 0, sampling_metadata={
                        "sampling_method": "inherited_only", "sampling_thinning": None,
                        "sampling_pilot_length": 0, "sampling_covariance_condition_number": None,
                        "sampling_warnings": ()})
                    continue
                x0 = X[int(self._rng.integers(0, n_inh))]
                if self.isotropic_sampling and bool(job.region.contains(x0, tol=sp.feasibility_tol)[0]):
                    seeds = (self._next_seed(), self._next_seed())
                else:  # an infeasible start fails in the pilot call, before the main seed
                    seeds = (self._next_seed(), None)
                reqs.append((job, X, y, n_inh, n_new, x0, seeds))
            if not reqs:
                return
            regions = [r[0].region for r in reqs]
            metas = [{"sampling_method": type(sp).__name__, "sampling_thinning": sp.thinning,
                      "sampling_pilot_length": 0, "sampling_covariance_condition_number": None,
                      "sampling_warnings": ()} for _ in reqs]
            if not self.isotropic_sampling:
                out = sp.sample_many(regions, [r[4] for r in reqs], [r[6][0] for r in reqs], [r[5] for r in reqs])
            else:
                # covariance-shaped top-ups (builder.py:1141-1200): every child's
                # pilot chain in one launch, its spectrum on the host, then every
                # main chain in one launch with its own direction map
                pilot_len = self.isotropic_pilot_multiplier * self.dimension
                pilot_sampler = replace(sp, burn_in=0, thinning=1, direction_eigenvectors=None,
                                        direction_eigenvalues=None)
                pilots = pilot_sampler.sample_many(regions, [pilot_len] * len(reqs), [r[6][0] for r in reqs],
                                                   [r[5] for r in reqs])
                out = [None] * len(reqs)
                main_idx, spectra, starts = [], [], []
                good = [q for q, pl in enumerate(pilots) if not isinstance(pl, Exception)
                        and np.asarray(pl, float).shape == (pilot_len, self.dimension)]
                eig = dict(zip(good, self._pilot_spectra([np.asarray(pilots[q], float) for q in good], sp)))
                for q, pilot in enumerate(pilots):
                    if isinstance(pilot, Exception):
                        if reqs[q][6][1] is not None:  # failed after the main seed was drawn: undo
                            self._rng.bit_generator.state = rng_state
                            self.oracle_queries = queries0
                            for j, smp in saved:
                                j.topped, j.topup_error, j.topup_pending, j.samples = False, None, None, smp
                            return
                        out[q] = pilot
                        continue
                    pilot = np.asarray(pilot, float)
                    if pilot.shape != (pilot_len, self.dimension):
                        out[q] = RuntimeError(f"Pilot sampler returned shape {pilot.shape}.")
                        continue
                    vecs, vals = eig[q]
                    safe, floor = floor_covariance_eigenvalues(vals, sp.direction_eigenvalue_floor)
                    saturated = bool(np.any(vals <= floor))
                    metas[q] = {"sampling_method": "isotropic_hit_and_run", "sampling_thinning": sp.thinning,
                                "sampling_pilot_length": pilot_len,
                                "sampling_covariance_condition_number": float(np.max(safe) / np.min(safe)),
                                "sampling_covariance_eigenvalue_floor": floor,
                                "sampling_covariance_floor_saturated": saturated,
                                "sampling_warnings": ("covariance_eigenvalue_floor_saturated",) if saturated else ()}
                    main_idx.append(q)
                    spectra.append((vecs, vals))
                    starts.append(pilot[-1])
                if main_idx:
                    mains = sp.sample_many([regions[q] for q in main_idx], [reqs[q][4] for q in main_idx],
                                           [reqs[q][6][1] for q in main_idx], starts, spectra=spectra)
                    for q, X_new in zip(main_idx, mains):
                        out[q] = X_new
            for q, ((job, X, y, n_inh, n_new, x0, seeds), X_new) in enumerate(zip(reqs, out)):
                meta = metas[q]
                if isinstance(X_new, Exception):
                    job.topup_error = X_new
                    continue
                if X_new.shape != (n_new, self.dimension):
                    job.topup_error = RuntimeError(f"Sampler returned shape {X_new.shape}; expected "
                                                   f"{(n_new, self.dimension)}.")
                    continue
                if not np.all(job.region.contains(X_new)):
                    job.topup_error = RuntimeError("Sampler returned points outside the region.")
                    continue
                job.topup_pending = (X, y, n_inh, n_new, X_new, dict(meta))
        for job, *_ in reqs:
            pend = getattr(job, "topup_pending", None)
            if pend is None or job.topup_error is not None:
                continue
            X, y, n_inh, n_new, X_new, m = pend
            job.topup_pending = None
            try:
                y_new = self._query_oracle(X_new)
            except (RuntimeError, ValueError) as exc:
                job.topup_error = exc
                continue
            job.samples = _NodeSamples(np.vstack([X, X_new]), np.concatenate([y, y_new]), n_inh, n_new, m)

    def _top_up_child(self, region, inherited_X, inherited_y) -> _NodeSamples:
        """builder.py:502-551"""

        X = np.asarray(inherited_X, dtype=float)
        y = np.asarray(inherited_y, dtype=float).reshape(-1)
        if X.shape[0] == 0:
            raise RuntimeError("Cannot seed child sampling without an inherited point.")
        if X.shape[0] > self._target_samples:
            keep = self._rng.choice(X.shape[0], size=self._target_samples, replace=False)
            X, y = X[keep], y[keep]
        n_inh = X.shape[0]
        n_new = self._target_samples - n_inh
        if n_new == 0:
            return _NodeSamples(X, y, n_inh, 0, sampling_metadata={
                "sampling_method": "inherited_only", "sampling_thinning": None, "sampling_pilot_length": 0,
                "sampling_covariance_condition_number": None, "sampling_warnings": ()})
        x0 = X[int(self._rng.integers(0, n_inh))]
        X_new, meta = self._sample_region(region, n_new, x0=x0, sampler=self.sampler)
        y_new = self._query_oracle(X_new)
        return _NodeSamples(np.vstack([X, X_new]), np.concatenate([y, y_new]), n_inh, n_new, meta)

    # ---------------------------------------------------------------- splits
    def _fit_split(self, X, y, parent_model, parent_mse, depth, prepared):
        state = self._split_state(X, y, depth, prepared)
        while True:
            try:
                result = self._run_splitter(X, y, parent_model, parent_mse, state.temperature, prepared,
                                            min_side_fallback=state.fallback)
            except SplitNotFoundError as exc:
                result = exc
            if self._retry_split(state, result):
                continue
            if isinstance(result, SplitNotFoundError):
                raise state.error(result) from result
            return result, state.context, state.metadata

    def _split_state(self, X, y, depth, prepared) -> _SplitState:
        temperature, context, tuned = self._resolve_split_temperature(X, y, depth, prepared)
        return _SplitState(temperature, context, 0 if tuned else self.max_retries_on_failure,
                           bool(getattr(self.splitter, "min_side_fallback", False)))

    def _retry_split(self, state: _SplitState, result) -> bool:
        """Retry min-side failures or rejected gains (builder.py:626-638)."""

        failed = isinstance(result, SplitNotFoundError)
        reason = result.reason if failed else self._split_rejection_reason(result)
        if reason is not None:
            state.reasons.append(reason)
        eligible = (reason == "min_side_points" if failed
                    else reason in ("insufficient_split_gain", "insufficient_relative_split_gain"))
        if eligible and state.retries < state.limit:
            state.retries += 1
            self.restarts_on_failure += 1
            return True
        return False

    def _resolve_split_temperature(self, X, y, depth, prepared):
        """builder.py:640-682"""

        config = self.temperature_config
        if config is None or config.strategy == "splitter":
            return None, {"temperature": getattr(self.splitter, "temperature", None), "temperature_c": None,
                          "temperature_tuned_at_node": False}, False
        scores = None
        if config.strategy == "fixed":
            c, tuned = config.c, False
        elif config.strategy == "tune_root" and self._root_temperature_c is not None:
            c, tuned = self._root_temperature_c, False
        else:
            c, scores = self._tune_temperature(X, y, prepared)
            tuned = True
            if config.strategy == "tune_root" and depth == 0:
                self._root_temperature_c = c
        temperature = self._temperature_for_c(X, c)
        meta = {"temperature": temperature, "temperature_c": c, "temperature_scale_mode": config.scale_mode,
                "temperature_tuned_at_node": tuned}
        if self.store_diagnostics and tuned:
            meta["temperature_candidate_scores"] = scores
        return temperature, meta, tuned

    def _tune_temperature(self, X, y, prepared):
        """Grid of c on a held-out split of the node samples (builder.py:684-773)."""

        config = self.temperature_config
        n_val = max(1, int(round(config.validation_fraction * X.shape[0])))
        perm = self._rng.permutation(X.shape[0])
        val_idx, fit_idx = perm[:n_val], perm[n_val:]
        X_fit, y_fit, X_val, y_val = X[fit_idx], y[fit_idx], X[val_idx], y[val_idx]
        fit_design = None if prepared is None else prepared.subset(fit_idx)
        parent_model, parent_pred = self._fit_node_model(X_fit, y_fit, fit_design)
        parent_mse = mean_squared_error(y_fit, parent_pred)
        comparison_seed = self._next_seed()
        temperature_seed = self._next_seed()
        candidates, best = [], None
        temps = [self._temperature_for_c(X_fit, c, random_seed=temperature_seed) for c in config.c_values]
        batched = None
        if self.batched_temperature_tuning and fit_design is None and hasattr(self.splitter, "split_temperatures"):
            # every candidate starts from the same restarts (one seed): one
            # launch with a node per candidate gives each candidate's split
            s = copy.deepcopy(self.splitter)
            s.random_state = comparison_seed
            s._timing_profile = self._timing_profile
            with self._timing_context("splitter"):
                batched = s.split_temperatures(X_fit, y_fit, temps, parent_model, parent_mse,
                                               hard_refit=self.hard_refits)
        for i, (c, T) in enumerate(zip(config.c_values, temps)):
            try:
                if batched is not None:
                    if isinstance(batched[i], SplitNotFoundError):
                        raise batched[i]
                    result = batched[i]
                else:
                    result = self._run_splitter(X_fit, y_fit, parent_model, parent_mse, T, fit_design,
                                                random_seed=comparison_seed)
            except SplitNotFoundError as exc:
                candidates.append({"c": c, "temperature": T, "validation_mse": np.inf, "failure_reason": exc.reason})
                continue
            rejection = self._split_rejection_reason(result)
            if rejection is not None:
                candidates.append({"c": c, "temperature": T, "validation_mse": np.inf, "failure_reason": rejection})
                continue
            mse = mean_squared_error(y_val, result.predict(X_val))
            candidates.append({"c": c, "temperature": T, "validation_mse": mse, "failure_reason": None})
            if best is None or mse < best[0]:
                best = (mse, float(c))
        if best is None:
            raise SplitNotFoundError("temperature_tuning_failed",
                                     "All temperature candidates failed to produce a valid split.")
        return best[1], candidates

    def _run_splitter(self, X, y, parent_model, parent_mse, temperature, prepared, random_seed=None,
                      min_side_fallback=None):
        """builder.py:775-823: a fresh splitter copy per attempt, seeded from the build stream."""

        s = copy.deepcopy(self.splitter)
        if temperature is not None:
            s.temperature = float(temperature)
        if min_side_fallback is not None:
            s.min_side_fallback = min_side_fallback
        s.random_state = self._next_seed() if random_seed is None else random_seed
        s._timing_profile = self._timing_profile
        kwargs = {"parent_model": parent_model, "parent_loss": parent_mse}
        if not self.hard_refits:
            kwargs["hard_refit"] = False
        with self._timing_context("splitter"):
            return s.split(X, y, **kwargs)

    def _split_rejection_reason(self, result: SplitResult) -> str | None:
        """builder.py:463-483"""

        values = [result.parent_loss, result.z, *result.w]
        if result.has_hard_fit:
            values.extend((result.loss, result.split_gain, result.relative_split_gain))
        elif self.check_split_gain:
            raise ValueError("Split-gain checks require final hard refits.")
        if not np.all(np.isfinite(values)):
            return "nonfinite_split"
        if self.check_split_gain and result.split_gain <= self.min_split_gain:
            return "insufficient_split_gain"
        if self.check_split_gain and result.relative_split_gain <= self.min_relative_split_gain:
            return "insufficient_relative_split_gain"
        if result.stop_reason in ("line_search_failed", "max_line_search_failures", "alpha_min_reached",
                                  "non_descent_direction") and result.n_iters == 0:
            return "optimizer_failed_without_progress"
        return None

    def _split_warnings(self, result: SplitResult) -> tuple[str, ...]:
        w = []
        if result.n_iters == 0 and result.stop_reason == "gradient_tolerance":
            w.append("small_init_grad")
        if not result.converged:
            w.append(result.stop_reason)
        for key in ("alpha_min_saturated", "alpha_max_saturated", "high_model_conditioning", "min_side_fallback"):
            if bool(result.metadata.get(key, False)):
                w.append(key)
        return tuple(dict.fromkeys(w))

    def _diagnostic_warnings(self, diagnostics) -> tuple[str, ...]:
        if diagnostics is None:
            return ()
        w = []
        if diagnostics.get("n_iters") == 0 and diagnostics.get("stop_reason") == "gradient_tolerance":
            w.append("small_init_grad")
        if bool(diagnostics.get("high_model_conditioning", False)):
            w.append("high_model_conditioning")
        return tuple(w)

    @staticmethod
    def _combine_warnings(*groups) -> tuple[str, ...]:
        return tuple(dict.fromkeys(w for g in groups for w in g))

    def _split_summary(self, result: SplitResult) -> dict[str, object]:
        return {"hard_refit": result.has_hard_fit, "split_mse": result.loss, "split_gain_mse": result.split_gain,
                "relative_split_gain_mse": result.relative_split_gain, "split_n_left": result.n_left,
                "split_n_right": result.n_right, "split_converged": result.converged,
                "split_stop_reason": result.stop_reason, "split_iterations": result.n_iters}

    # ---------------------------------------------------------------- fits
    def _prepare_design(self, X):
        if isinstance(self.model_template, PolynomialRidgeModel) and self.model_template.degree > 2:
            return self.model_template.prepare_design(X)
        return None  # features are generated on chip from X

    def _fit_node_model(self, X, y, prepared):
        if prepared is None and self.fit_precision == "mixed":
            from .models import fit_models_batched

            with self._timing_context("model_refit"):
                model = fit_models_batched(self.model_template, [X], [y], precision="mixed")[0]
                if isinstance(model, Exception):
                    raise model
                return model, model.predict(X)
        model = self.model_template.clone()
        with self._timing_context("model_refit"):
            if prepared is None:
                model.fit(X, y)
                return model, model.predict(X)
            model.fit_design(prepared, y)
            return model, model.predict_design(prepared)

    def _fit_cohort(self, jobs) -> None:
        """Fit the node models of a BFS cohort in one batched solve.

        Each job whose samples are final (the root, or a child whose cohort
        top-up succeeded) gets ``fit_cache``: the model and its predictions
        that ``_fit_node_model`` would return, or the exception it would
        raise.  Jobs that still need their own top-up, validation fits or a
        host design matrix keep the per-node path.  The solves are the
        single-node solves, batched, so the tree does not change.
        """

        if not self.batched_fits or self.validation_fraction > 0.0:
            return
        if isinstance(self.model_template, PolynomialRidgeModel) and self.model_template.degree > 2:
            return
        ready = [j for j in jobs if j.fit_cache is None and (
            j.parent is None or (j.topped and j.topup_error is None and j.topup_pending is None))]
        if len(ready) < 2:
            return
        from .models import fit_models_batched

        with self._timing_context("model_refit"):
            models = fit_models_batched(self.model_template, [j.samples.X for j in ready],
                                        [j.samples.y for j in ready], precision=self.fit_precision)
            for j, m in zip(ready, models):
                j.fit_cache = (m, None) if isinstance(m, Exception) else (m, m.predict(j.samples.X))

    def _fit_convergence_model(self, X, y, prepared):
        n_val = min(max(1, int(round(self.validation_fraction * X.shape[0]))), X.shape[0] - 1)
        fit_idx = self._rng.permutation(X.shape[0])[n_val:]
        design = None if prepared is None else prepared.subset(fit_idx)
        model, _ = self._fit_node_model(X[fit_idx], y[fit_idx], design)
        pred = model.predict(X) if prepared is None else model.predict_design(prepared)
        return model, pred, fit_idx.size

    def _fit_full_node_model(self, samples, prepared, extra_metadata=None, cached=None):
        if cached is not None:
            model, pred = cached
            if isinstance(model, Exception):
                raise model
        else:
            model, pred = self._fit_node_model(samples.X, samples.y, prepared)
        fit_error = float(self.error_metric(samples.y, pred))
        fit_mse = mean_squared_error(samples.y, pred)
        meta = self._node_metadata(samples, fit_error, fit_mse, model)
        if extra_metadata is not None:
            meta.update(extra_metadata)
        return model, fit_error, fit_mse, meta

    def _temperature_for_c(self, X, c, random_seed=None) -> float:
        cfg = self.temperature_config
        method = cfg.nn_method
        if method is None:
            method = "bruteforce" if self.dimension >= cfg.bruteforce_dimension_threshold else "kdtree"
        return estimate_temperature(X, mode=cfg.scale_mode, c=c, max_points=cfg.max_points,
                                    random_state=self._next_seed() if random_seed is None else random_seed,
                                    nn_method=method)

    def _node_metadata(self, samples, fit_error, fit_mse, model) -> dict[str, object]:
        solve = ridge_solve_diagnostics(model)
        cond = None if solve is None else solve.get("cond_estimate")
        warnings = (("high_model_conditioning",) if cond is not None and float(cond) >= MODEL_CONDITION_WARNING_THRESHOLD
                    else ())
        g = (lambda k: None if solve is None else solve.get(k))
        return {"fit_error": fit_error, "fit_error_metric": self._metric_name(), "fit_mse": fit_mse,
                "n_samples": samples.X.shape[0], "n_inherited": samples.n_inherited, "n_new": samples.n_new,
                "fit_solver_requested": g("solver_requested"), "fit_solver_used": g("solver_used"),
                "fit_condition_estimator": g("condition_estimator"), "fit_cond_estimate": cond,
                "fit_ridge_effective": g("ridge_effective"), "fit_rank": g("rank"),
                "fit_fallback_reason": g("fallback_reason"), "warnings": warnings, **samples.sampling_metadata}

    def _make_leaf(self, model, region, depth, node_id, status, metadata, samples) -> LeafNode:
        if getattr(self, "_leaf_samples", None) is not None:
            self._leaf_samples[node_id] = samples
        meta = dict(metadata)
        if self.store_leaf_representative:
            meta["sample_centroid"] = np.mean(samples.X, axis=0)
        self._store_samples(meta, samples)
        return LeafNode(model=model, region=region, depth=depth, node_id=node_id, status=status, metadata=meta)

    def _store_samples(self, metadata, samples) -> None:
        if self.store_samples:
            metadata["X"] = samples.X.copy()
            metadata["y"] = samples.y.copy()

    # ---------------------------------------------------------------- sampling
    def _sample_root(self, region):
        if isinstance(self.domain, BoxDomain) and self.exact_box_root:
            with self._timing_context("sampling"):
                X = sample_uniform_box(self.domain.bounds, self._target_samples, random_state=self._next_seed())
            return X, {"sampling_method": "exact_uniform_box", "sampling_thinning": None, "sampling_pilot_length": 0,
                       "sampling_covariance_condition_number": None, "sampling_warnings": ()}
        return self._sample_region(region, self._target_samples, x0=None, sampler=self.root_sampler)

    def _pilot_spectra(self, pilots, sampler):
        """(eigenvectors, eigenvalues) of each pilot's sample covariance
        (builder.py:1141-1200): on the host with numpy's eigh when the sampler
        follows the reference's random stream, else all pilots in one device
        launch (``art_covariance_eigh``), so covariance-shaped top-ups stay on
        the GPU; one-at-a-time and cohort top-ups take the same path."""

        if getattr(sampler, "rng_mode", "reference") == "device":
            return covariance_eigendecomposition_batched(pilots)
        return [sample_covariance_eigendecomposition(p) for p in pilots]

    def _sample_region(self, region, n, *, x0, sampler):
        with self._timing_context("sampling"):
            return self._sample_region_untimed(region, n, x0=x0, sampler=sampler)

    def _sample_region_untimed(self, region, n, *, x0, sampler):
        """Plain or covariance-shaped hit-and-run (builder.py:1116-1208)."""

        if not self.isotropic_sampling:
            X = np.asarray(sampler.sample(region, n, random_state=self._next_seed(), x0=x0), dtype=float)
            meta = {"sampling_method": type(sampler).__name__, "sampling_thinning": getattr(sampler, "thinning", None),
                    "sampling_pilot_length": 0, "sampling_covariance_condition_number": None, "sampling_warnings": ()}
        else:
            pilot_len = self.isotropic_pilot_multiplier * self.dimension
            pilot_sampler = replace(sampler, burn_in=0, thinning=1, direction_eigenvectors=None,
                                    direction_eigenvalues=None)
            pilot = np.asarray(pilot_sampler.sample(region, pilot_len, random_state=self._next_seed(), x0=x0), float)
            if pilot.shape != (pilot_len, self.dimension):
                raise RuntimeError(f"Pilot sampler returned shape {pilot.shape}.")
            vecs, vals = self._pilot_spectra([pilot], sampler)[0]
            safe, floor = floor_covariance_eigenvalues(vals, sampler.direction_eigenvalue_floor)
            saturated = bool(np.any(vals <= floor))
            node_sampler = replace(sampler, direction_eigenvectors=vecs, direction_eigenvalues=vals)
            X = np.asarray(node_sampler.sample(region, n, random_state=self._next_seed(), x0=pilot[-1]), float)
            meta = {"sampling_method": "isotropic_hit_and_run", "sampling_thinning": sampler.thinning,
                    "sampling_pilot_length": pilot_len,
                    "sampling_covariance_condition_number": float(np.max(safe) / np.min(safe)),
                    "sampling_covariance_eigenvalue_floor": floor, "sampling_covariance_floor_saturated": saturated,
                    "sampling_warnings": ("covariance_eigenvalue_floor_saturated",) if saturated else ()}
        if X.shape != (n, self.dimension):
            raise RuntimeError(f"Sampler returned shape {X.shape}; expected {(n, self.dimension)}.")
        if not np.all(region.contains(X)):
            raise RuntimeError("Sampler returned points outside the region.")
        return X, meta

    # ---------------------------------------------------------------- misc
    def _timing_context(self, category: BuildTimingCategory):
        return nullcontext() if self._timing_profile is None else self._timing_profile.measure(category)

    def _query_oracle(self, X) -> np.ndarray:
        X = np.asarray(X, dtype=float)
        if self.oracle_vectorized:
            values = np.asarray(self.oracle(X), dtype=float).reshape(-1)
            if values.shape[0] != X.shape[0]:
                raise ValueError("A vectorized oracle must return one value per input row.")
            self.oracle_queries += X.shape[0]
            return values
        values = np.empty(X.shape[0])
        for i, x in enumerate(X):
            values[i] = float(self.oracle(x))
            self.oracle_queries += 1
        return values

    def _resolve_effective_dimension(self):
        if self.sample_count is not None:
            try:
                return model_effective_dimension(self.model_template, self.dimension)
            except TypeError:
                return None
        return model_effective_dimension(self.model_template, self.dimension)

    def _resolve_sample_count(self) -> int:
        if self.sample_count is None:
            return self.sample_multiplier * int(self._effective_dimension)
        if callable(self.sample_count):
            return int(self.sample_count(self.model_template, self.dimension))
        return int(self.sample_count)

    def _metric_name(self) -> str:
        return getattr(self.error_metric, "__name__", type(self.error_metric).__name__)

    def _next_seed(self) -> int:
        return int(self._rng.integers(0, 2**31 - 1))


class LevelSplitDispatcher:
    """Split a whole BFS cohort in one ``art_split_level`` launch sequence.

    Follows BatchedSplitDispatcher (_cuda_batched_builder.py:38-95): the split
    state of every job is resolved first (in job order), then all first
    attempts run together; retries (fallback enabled on a job's last allowed
    attempt) run as further cohort calls.  Initial theta come from each
    attempt's splitter seed exactly as SoftObliqueSplitter.split draws them.
    """

    def __init__(self, builder: RegressionTreeBuilder):
        self.b = builder

    def __call__(self, ready: list[_NodeWork]) -> list[TreeNode]:
        from .splitters import level_result_to_split, split_level, _model_kind

        b = self.b
        nodes: list = [None] * len(ready)
        jobs, states, first_seeds = [], [], []
        for pos, job in enumerate(ready):
            try:
                st = b._split_state(job.samples.X, job.samples.y, job.depth, job.prepared)
            except SplitNotFoundError as exc:
                nodes[pos] = b._finish_node(job, exc)
                continue
            jobs.append((pos, job))
            states.append(st)
            first_seeds.append(b._next_seed())  # the scalar path's draw order: state, then seed
        outcomes = [None] * len(jobs)
        pending = list(range(len(jobs)))
        s0 = b.splitter
        kind = _model_kind(s0.model_template)
        R = max(1, s0.n_restarts)
        first = True
        while pending:
            seeds = first_seeds if first else [b._next_seed() for _ in pending]
            first = False
            with b._timing_context("splitter"):
                Xs, ys, ro, th0, temps, fb, parents, d = [], [], [0], [], [], [], [], b.dimension
                for j, seed in zip(pending, seeds):
                    job = jobs[j][1]
                    X, y = job.samples.X, job.samples.y
                    rng = np.random.default_rng(seed)
                    th0.append([s0._initialize_theta(X, rng) for _ in range(R)])
                    Xs.append(X.reshape(-1))
                    ys.append(y)
                    ro.append(ro[-1] + X.shape[0])
                    temps.append(s0.temperature if states[j].temperature is None else states[j].temperature)
                    fb.append(1 if states[j].fallback else 0)
                    parents.append(job.parent_mse)
                if b.cuda_graphs:
                    from .graphs import shared_split_graphs
                    from .models import kind_feature_count

                    res = shared_split_graphs().split_level(
                        s0, np.concatenate(Xs), np.concatenate(ys), ro, [d] * len(pending), [kind] * len(pending),
                        temps, s0.model_template.ridge, parent_loss=parents, min_side_fallback=fb,
                        theta0=np.array(th0), hard_refit=b.hard_refits, traces=b.store_diagnostics,
                        max_dim=d, max_features=kind_feature_count(d, kind))
                else:
                    res = split_level(s0, np.concatenate(Xs), np.concatenate(ys), ro, [d] * len(pending),
                                      [kind] * len(pending), temps, s0.model_template.ridge, parent_loss=parents,
                                      min_side_fallback=fb, theta0=np.array(th0), hard_refit=b.hard_refits,
                                      traces=b.store_diagnostics)
            again = []
            for q, j in enumerate(pending):
                job = jobs[j][1]
                s = copy.copy(s0)
                s.temperature = temps[q]
                try:
                    result = level_result_to_split(s, res, q, job.samples.X.shape[0], job.parent_mse, b.hard_refits)
                except SplitNotFoundError as exc:
                    result = exc
                if b._retry_split(states[j], result):
                    again.append(j)
                else:
                    outcomes[j] = result
            pending = again
        for (pos, job), st, result in zip(jobs, states, outcomes):
            if isinstance(result, SplitNotFoundError):
                nodes[pos] = b._finish_node(job, st.error(result))
            else:
                nodes[pos] = b._finish_node(job, result, {**st.context, **st.metadata})
        return nodes
