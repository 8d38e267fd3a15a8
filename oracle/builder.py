"""Oracle: depth-first tree build (reference art/builder.py) -- test
infrastructure only.

A numpy restatement of RegressionTreeBuilder.build with traversal="dfs" for
the configurations the benchmarks use: a box domain sampled exactly at the
root (builder.py:1072-1094), children that inherit the parent's samples on
their side and are topped up by the scalar HitAndRunSampler from one of them
(builder.py:502-551, sampling.py:445-495), affine or polynomial ridge node
models, relative L2 fit error against a threshold, a depth limit
(builder.py:358-400), and SoftObliqueSplitter splits with a fixed temperature
(TemperatureConfig(strategy="splitter"), builder.py:640-682) and hard refits
only when restarts need them (builder.py:264-269).  The builder's random
stream is consumed in the reference's order (builder.py:1250-1251), so with
the same random_state the tree equals the reference's.  Options outside this
subset (isotropic sampling, temperature tuning, retries, validation
fractions, gain checks) raise.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import ridge as R
from . import split as S


def relative_l2_error(y, pred, floor=1e-12):
    """metrics.py:36-43"""
    return float(np.linalg.norm(y - pred) / max(float(np.linalg.norm(y)), floor))


def step_interval(A, b, x, u, tol=1e-10):
    """HitAndRunSampler._step_interval (sampling.py:540-564)."""
    Ax, Au = A @ x, A @ u
    slack = b - Ax
    pos, neg = Au > 1e-14, Au < -1e-14
    if np.any(~(pos | neg) & (slack < -tol)):
        raise RuntimeError("Current point is infeasible for the hit-and-run step.")
    ratios = np.zeros_like(Au)
    np.divide(slack, Au, out=ratios, where=pos | neg)
    t_lo = np.max(ratios, where=neg, initial=-np.inf)
    t_hi = np.min(ratios, where=pos, initial=np.inf)
    if t_lo > t_hi:
        raise RuntimeError("Empty hit-and-run step interval.")
    return float(t_lo), float(t_hi)


def hit_and_run(A, b, x0, n, burn_in, thinning, seed):
    """HitAndRunSampler.sample with isotropic directions (sampling.py:445-495)."""
    rng = np.random.default_rng(seed)
    x = np.asarray(x0, float).copy()
    out = []
    for step in range(burn_in + n * thinning):
        u = rng.normal(size=x.shape[0])
        nrm = np.linalg.norm(u)
        if nrm == 0.0:
            continue
        u = u / nrm
        lo, hi = step_interval(A, b, x, u)
        x = x + rng.uniform(lo, hi) * u
        if step >= burn_in and (step - burn_in) % thinning == 0:
            out.append(x.copy())
    return np.asarray(out, float).reshape(-1, x.shape[0])


@dataclass
class Node:
    node_id: str
    depth: int
    status: str
    w: np.ndarray | None = None
    z: float | None = None
    coef: np.ndarray | None = None
    n_samples: int = 0
    left: "Node | None" = None
    right: "Node | None" = None
    fit_error: float = 0.0
    region: tuple | None = None        # (A, b) of a leaf, kept for refinement
    X: np.ndarray | None = None        # a leaf's samples, kept for refinement
    y: np.ndarray | None = None


@dataclass
class Builder:
    lo: np.ndarray
    hi: np.ndarray
    oracle: object
    kind: int
    ridge: float
    temperature: float
    error_threshold: float
    max_depth: int
    sample_count: int
    params: S.Params
    burn_in: int = 0
    thinning: int = 5
    random_state: int = 0
    refinement_rounds: int = 0
    refinement_points: int = 1024
    refinement_leaves: int = 4
    top_up: bool = True                # False: children keep only their inherited samples
    queries: int = field(default=0, init=False)

    def next_seed(self):
        return int(self.rng.integers(0, 2**31 - 1))

    def query(self, X):
        self.queries += X.shape[0]
        return np.asarray(self.oracle(X), float).reshape(-1)

    def build(self) -> Node:
        self.rng = np.random.default_rng(self.random_state)
        self.queries = 0
        d = self.lo.shape[0]
        A = np.vstack([np.eye(d), -np.eye(d)])                      # BoxDomain.as_region (domain.py:87-92)
        b = np.concatenate([self.hi, -self.lo])
        X = np.random.default_rng(self.next_seed()).uniform(self.lo, self.hi, size=(self.sample_count, d))
        y = self.query(X)
        root = self._node(A, b, X, y, 0, "root", parent=False)
        for _ in range(self.refinement_rounds):
            root = self._refine_round(root)
        return root

    def _refine_round(self, root):
        """The refinement round of the GPU builder (RegressionTreeBuilder._refine_round):
        the leaves of largest fit error get new hit-and-run samples and are
        rebuilt from all their samples through the node policy."""
        leaves = [n for n in iter_nodes(root) if n.left is None]
        order = sorted(range(len(leaves)), key=lambda i: -leaves[i].fit_error)
        chosen = [leaves[i] for i in order[: self.refinement_leaves]]
        base, extra = divmod(self.refinement_points, len(chosen))
        for q, leaf in enumerate(chosen):
            m = base + (1 if q < extra else 0)
            if m == 0:
                continue
            A, b, X, y = leaf.region[0], leaf.region[1], leaf.X, leaf.y
            x0 = X[int(self.rng.integers(0, X.shape[0]))]
            Xn = hit_and_run(A, b, x0, m, self.burn_in, self.thinning, self.next_seed())
            sub = self._node(A, b, np.vstack([X, Xn]), np.concatenate([y, self.query(Xn)]), leaf.depth,
                             leaf.node_id, parent=False)
            root = _replace(root, leaf, sub)
        return root

    def _fit(self, X, y):
        phi = R.features(X, self.kind)
        res = R.solve_weighted_ridge(phi, y, np.ones(len(y)), self.ridge)
        beta = res["coefficients"]
        high = res["cond_estimate"] is not None and float(res["cond_estimate"]) >= 1e10   # models.py:22
        return beta, phi @ beta, high

    def _warnings(self, res, high_cond):
        """_split_warnings and the node's conditioning warning (builder.py:944-958, 1006-1012)."""
        p = self.params
        return bool(high_cond
                    or (res["n_iters"] == 0 and res["stop_reason"] == "gradient_tolerance")
                    or not res["converged"]
                    or (p.adaptive_alpha and (res["final_alpha"] <= p.alpha_min or res["final_alpha"] >= p.alpha_max))
                    or res["fallback"])

    def _node(self, A, b, X, y, depth, node_id, parent=True) -> Node:
        if parent and self.top_up:                                      # _top_up_child (builder.py:502-551)
            if X.shape[0] > self.sample_count:
                keep = self.rng.choice(X.shape[0], size=self.sample_count, replace=False)
                X, y = X[keep], y[keep]
            n_new = self.sample_count - X.shape[0]
            if n_new > 0:
                x0 = X[int(self.rng.integers(0, X.shape[0]))]
                Xn = hit_and_run(A, b, x0, n_new, self.burn_in, self.thinning, self.next_seed())
                if not np.all(Xn @ A.T <= b[None, :] + 1e-10):
                    raise RuntimeError("Sampler returned points outside the region.")
                X, y = np.vstack([X, Xn]), np.concatenate([y, self.query(Xn)])
        beta, pred, high_cond = self._fit(X, y)
        err = relative_l2_error(y, pred)

        def leaf(status):
            return Node(node_id, depth, status, coef=beta, n_samples=len(y), fit_error=err, region=(A, b), X=X, y=y)

        if err <= self.error_threshold:
            return leaf("tolerance_met")
        if depth >= self.max_depth:
            return leaf("max_depth")
        parent_mse = float(np.mean((y - pred) ** 2))
        hard = self.params.n_restarts != 1                               # builder.py:264-269
        split_rng = np.random.default_rng(self.next_seed())              # _run_splitter random_state
        starts = [S.initialize_theta(X, split_rng) for _ in range(max(1, self.params.n_restarts))]
        try:
            res = S.split(X, y, starts, self.temperature, self.kind, self.ridge, parent_mse, self.params,
                          hard_refit=hard)
        except ValueError as exc:
            return leaf(str(exc))
        failures = ("line_search_failed", "max_line_search_failures", "alpha_min_reached", "non_descent_direction")
        if not np.all(np.isfinite(np.r_[res["w"], res["z"]])):
            return leaf("nonfinite_split")
        if res["stop_reason"] in failures and res["n_iters"] == 0:
            return leaf("optimizer_failed_without_progress")
        w, z = res["w"], float(res["z"])
        node = Node(node_id, depth, "split_with_warnings" if self._warnings(res, high_cond) else "split", w=w, z=z,
                    n_samples=len(y))
        right = (X @ w - z) >= 0.0                                       # builder.py:494
        node.left = self._node(np.vstack([A, w]), np.r_[b, z], X[~right], y[~right], depth + 1, f"{node_id}/L")
        node.right = self._node(np.vstack([A, -w]), np.r_[b, -z], X[right], y[right], depth + 1, f"{node_id}/R")
        return node


def _replace(root: Node, old: Node, new: Node) -> Node:
    if root is old:
        return new
    for n in iter_nodes(root):
        if n.left is old:
            n.left = new
        elif n.right is old:
            n.right = new
    return root


def iter_nodes(node: Node):
    """Pre-order walk (tree.py:212-221 order: node, left subtree, right subtree)."""
    yield node
    if node.left is not None:
        yield from iter_nodes(node.left)
    if node.right is not None:
        yield from iter_nodes(node.right)


def predict(root: Node, X, kind):
    out = np.empty(X.shape[0])
    for i, x in enumerate(X):
        n = root
        while n.left is not None:
            n = n.right if float(x @ n.w - n.z) >= 0.0 else n.left
        out[i] = float(R.features(x[None, :], kind)[0] @ n.coef)
    return out
