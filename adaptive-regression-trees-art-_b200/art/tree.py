"""Regression tree artifact and prediction (reference art/tree.py:15-241).

``RegressionTree.predict`` routes all points on the GPU (``art_tree_predict``):
the tree is flattened to child/plane/coefficient arrays and every point walks
it independently, with the side decided by the sign of the exact value of
w . x - z (>= 0 goes right; compensated and, near the plane, exact
expansion arithmetic on the device).  Save/load keep the reference's joblib artifact
(type "art.regression_tree", version 1).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any, Iterator, Mapping, Optional, Union

import numpy as np

from .domain import PolytopeRegion
from .models import AffineRidgeModel, PolynomialRidgeModel, RegressionModel, kind_feature_count

TREE_ARTIFACT_TYPE = "art.regression_tree"
TREE_ARTIFACT_VERSION = 1


@dataclass
class LeafNode:
    model: RegressionModel
    region: Optional[PolytopeRegion] = None
    depth: int = 0
    node_id: str = "root"
    status: str = "leaf"
    metadata: dict[str, Any] = field(default_factory=dict)

    def predict_one(self, x: np.ndarray) -> float:
        return float(self.model.predict(np.asarray(x, dtype=float).reshape(1, -1))[0])


TreeNode = Union["SplitNode", LeafNode]


@dataclass
class SplitNode:
    w: np.ndarray
    z: float
    left: TreeNode
    right: TreeNode
    region: Optional[PolytopeRegion] = None
    depth: int = 0
    node_id: str = "root"
    status: str = "split"
    metadata: dict[str, Any] = field(default_factory=dict)

    def __post_init__(self) -> None:
        self.w = np.asarray(self.w, dtype=float).reshape(-1)
        self.z = float(self.z)

    def route(self, x: np.ndarray) -> TreeNode:
        x = np.asarray(x, dtype=float).reshape(-1)
        if x.shape[0] != self.w.shape[0]:
            raise ValueError(f"x must have shape ({self.w.shape[0]},), got {x.shape}.")
        return self.right if float(self.w @ x - self.z) >= 0.0 else self.left


def _leaf_kind(model) -> int:
    from . import _native as N

    if type(model) is AffineRidgeModel:
        return N.FEATURES_AFFINE
    if type(model) is PolynomialRidgeModel and model.degree in (1, 2):
        return model.kind()
    return -1


class RegressionTree:
    """Prediction-only regression tree."""

    def __init__(self, root: Optional[TreeNode] = None, oracle_queries: int = 0,
                 metadata: Optional[dict[str, Any]] = None):
        self.root = root
        self.oracle_queries = int(oracle_queries)
        self.metadata = {} if metadata is None else dict(metadata)
        self._flat = None

    def __getstate__(self):
        state = dict(self.__dict__)
        state["_flat"] = None
        return state

    def save(self, path: str | Path, run_config: Mapping[str, Any] | None = None, compress: int = 3) -> Path:
        import joblib

        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        joblib.dump({"artifact_type": TREE_ARTIFACT_TYPE, "format_version": TREE_ARTIFACT_VERSION,
                     "tree": self, "run_config": {} if run_config is None else dict(run_config)},
                    path, compress=compress)
        return path

    @classmethod
    def load(cls, path: str | Path) -> tuple["RegressionTree", dict[str, Any]]:
        import joblib

        path = Path(path)
        artifact = joblib.load(path)
        if not isinstance(artifact, dict):
            raise TypeError(f"{path} is not a regression-tree artifact.")
        if artifact.get("artifact_type") != TREE_ARTIFACT_TYPE:
            raise ValueError(f"{path} has an unrecognized artifact type.")
        version = artifact.get("format_version")
        if version != TREE_ARTIFACT_VERSION:
            raise ValueError(f"Unsupported tree artifact version {version!r}; expected {TREE_ARTIFACT_VERSION}.")
        tree = artifact.get("tree")
        if not isinstance(tree, cls):
            raise TypeError(f"{path} does not contain a RegressionTree.")
        run_config = artifact.get("run_config", {})
        if not isinstance(run_config, dict):
            raise TypeError(f"{path} contains an invalid run configuration.")
        return tree, run_config

    # ----------------------------------------------------------- device form
    def flatten(self):
        """Flat arrays for the device walk: child[n,2], theta[n,d+1], coef, features."""

        if self._flat is not None:
            return self._flat
        nodes = list(self.iter_nodes())
        index = {id(n): i for i, n in enumerate(nodes)}
        d = None
        for n in nodes:
            if isinstance(n, SplitNode):
                d = n.w.shape[0]
                break
        if d is None:
            coef = getattr(self.root.model, "coef_", None)
            kind = _leaf_kind(self.root.model)
            d = (len(coef) - 1) if kind in (0, 1) else None
        child = np.full((len(nodes), 2), -1, dtype=np.int32)
        theta = np.zeros((len(nodes), (d or 1) + 1))
        kinds = np.zeros(len(nodes), dtype=np.int32)
        pmax = 1
        for n in nodes:
            if isinstance(n, LeafNode):
                c = getattr(n.model, "coef_", None)
                pmax = max(pmax, len(c) if c is not None else 1)
        coef = np.zeros((len(nodes), pmax))
        supported = True
        for i, n in enumerate(nodes):
            if isinstance(n, SplitNode):
                child[i] = (index[id(n.left)], index[id(n.right)])
                theta[i, :d] = n.w
                theta[i, d] = n.z
            else:
                k = _leaf_kind(n.model)
                c = getattr(n.model, "coef_", None)
                if k < 0 or c is None:
                    supported = False
                    continue
                kinds[i] = k
                coef[i, : len(c)] = c
        self._flat = (child, theta, coef, kinds, d, supported)
        return self._flat

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.asarray(X, dtype=float)
        if X.ndim == 1:
            X = X.reshape(1, -1)
        if X.ndim != 2:
            raise ValueError(f"X must have shape (n, d), got {X.shape}.")
        if X.shape[0] == 0:
            return np.empty(0, dtype=float)
        if self.root is None:
            raise ValueError("Tree has no root node.")
        leaf, pred = self.predict_device(X)
        return pred

    def predict_device(self, X, stream=None):
        """(leaf index, prediction) for every row of X, computed on the GPU."""

        from . import _native as N
        from ._device import ptr, require_cuda, stream_handle, to_device, torch

        child, theta, coef, kinds, d, supported = self.flatten()
        if not supported:
            raise TypeError("device prediction supports affine and degree 1/2 polynomial leaf models")
        if X.shape[1] != d:
            raise ValueError(f"X must have {d} columns, got {X.shape[1]}.")
        t = torch()
        dev = require_cuda()
        xs = to_device(np.ascontiguousarray(X), t.float64, dev)
        tensors = [to_device(a, dt, dev) for a, dt in ((child, t.int32), (theta, t.float64), (coef, t.float64),
                                                       (kinds, t.int32))]
        leaf = t.empty(X.shape[0], dtype=t.int32, device=dev)
        pred = t.empty(X.shape[0], dtype=t.float64, device=dev)
        lib = N.load_library()
        N.check(lib.art_tree_predict(int(d), child.shape[0], ptr(tensors[0]), ptr(tensors[1]), theta.shape[1],
                                     ptr(tensors[2]), coef.shape[1], ptr(tensors[3]), X.shape[0], ptr(xs),
                                     ptr(leaf), ptr(pred), stream_handle(stream)), "art_tree_predict")
        return leaf.cpu().numpy(), pred.cpu().numpy()

    def predict_one(self, x: np.ndarray) -> float:
        return self.leaf_for_point(x).predict_one(x)

    def leaf_for_point(self, x: np.ndarray) -> LeafNode:
        if self.root is None:
            raise ValueError("Tree has no root node.")
        node = self.root
        while isinstance(node, SplitNode):
            node = node.route(x)
        return node

    def iter_nodes(self) -> Iterator[TreeNode]:
        """Depth-first, left-to-right."""
        if self.root is None:
            return
        stack = [self.root]
        while stack:
            node = stack.pop()
            yield node
            if isinstance(node, SplitNode):
                stack.extend([node.right, node.left])

    def iter_leaves(self) -> Iterator[LeafNode]:
        for node in self.iter_nodes():
            if isinstance(node, LeafNode):
                yield node

    def path_to_node(self, node_id: str) -> tuple[TreeNode, ...]:
        if not isinstance(node_id, str) or not node_id:
            raise ValueError("node_id must be a nonempty string.")
        if self.root is None:
            raise KeyError(f"Tree does not contain a node with id {node_id!r}.")
        if node_id == self.root.node_id:
            return (self.root,)
        prefix = f"{self.root.node_id}/"
        if not node_id.startswith(prefix):
            raise KeyError(f"Tree does not contain a node with id {node_id!r}.")
        path: list[TreeNode] = [self.root]
        node = self.root
        for branch in node_id[len(prefix):].split("/"):
            if branch not in ("L", "R") or not isinstance(node, SplitNode):
                raise KeyError(f"Tree does not contain a node with id {node_id!r}.")
            node = node.left if branch == "L" else node.right
            path.append(node)
        if node.node_id != node_id:
            raise KeyError(f"Tree does not contain a node with id {node_id!r}.")
        return tuple(path)

    def get_node(self, node_id: str) -> TreeNode:
        return self.path_to_node(node_id)[-1]

    def num_nodes(self) -> int:
        return sum(1 for _ in self.iter_nodes())

    def num_split_nodes(self) -> int:
        return sum(isinstance(n, SplitNode) for n in self.iter_nodes())

    def num_leaves(self) -> int:
        return sum(1 for _ in self.iter_leaves())

    def max_depth(self) -> int:
        def depth(n):
            return n.depth if isinstance(n, LeafNode) else max(depth(n.left), depth(n.right))

        return 0 if self.root is None else depth(self.root)


def partition_rows(x, row_offsets, dims, theta, *, split=None, x_offsets=None, stream=None):
    """Stable node-sorted partition of every segment's rows by its plane, on the GPU.

    Segment k owns rows ``row_offsets[k]:row_offsets[k+1]`` (inputs at
    ``x_offsets[k]``, ``dims[k]`` columns) and is split by
    ``theta[k] = [w, z]``: a row goes right when the exact value of
    w . x - z is >= 0 (builder.py:487-500).  Returns ``(perm, n_right)`` as
    device tensors: perm lists, per segment, its left rows then its right
    rows (global row indices, input order kept on each side); segments with
    ``split[k] == 0`` keep their rows (all left, n_right 0).
    """

    from . import _native as N
    from ._device import ptr, require_cuda, stream_handle, to_device, torch

    t = torch()
    dev = require_cuda()
    lib = N.load_library()
    ro = to_device(row_offsets, t.int64, dev)
    dd = to_device(dims, t.int32, dev)
    K = int(dd.numel())
    xo = to_device(ro[:-1] * dd.to(t.int64) if x_offsets is None else x_offsets, t.int64, dev)
    xs = to_device(x, t.float64, dev)
    th = to_device(theta, t.float64, dev)
    if th.dim() != 2 or th.shape[0] != K:
        raise ValueError("theta must have shape (K, d_max + 1)")
    sp = None if split is None else to_device(np.asarray(split, np.int8) if not isinstance(split, t.Tensor) else split,
                                              t.int8, dev)
    kinds = t.zeros(K, dtype=t.int32, device=dev)
    total = int(ro[-1].item()) if K else 0
    perm = t.empty(max(total, 1), dtype=t.int64, device=dev)
    n_right = t.empty(max(K, 1), dtype=t.int32, device=dev)
    if K:
        seg = N.ArtSegments(K, ptr(ro), ptr(xo), ptr(dd), ptr(kinds))
        N.check(lib.art_partition_rows(C.byref(seg), ptr(xs), ptr(th), int(th.shape[1]), ptr(sp), ptr(perm),
                                       ptr(n_right), stream_handle(stream)), "art_partition_rows")
    perm, n_right = perm[:total], n_right[:K]
    perm._keepalive = (ro, dd, xo, xs, th, sp, kinds)
    return perm, n_right
