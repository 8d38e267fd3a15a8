"""Seeded synthetic workloads with the shapes and value distributions of the
ART hot-path benchmark configurations (no public dataset is involved).

``ridge_systems``   -- batched weighted ridge: 65,536 systems, n log-uniform
                       in [64, 8192], d in {8, 16}, affine or full quadratic
                       features, sigmoid-product weights, noisy quadratic y,
                       log-uniform ridge in [1e-8, 1e-2].
``split_nodes``     -- batched soft oblique split search nodes.
``polytopes``       -- box [-1,1]^d cut by random halfspaces with a
                       Chebyshev ball of radius >= 0.05.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from .models import kind_feature_count

# (d, feature kind) of the four ridge classes: p = 9, 17, 45, 153
RIDGE_CLASSES = ((8, N.FEATURES_AFFINE), (16, N.FEATURES_AFFINE), (8, N.FEATURES_POLY2),
                 (16, N.FEATURES_POLY2))


@dataclass
class RidgeWorkload:
    """Segmented inputs: x (sum n_k*d_k,), y, w (sum n_k,), CSR row offsets."""

    x: object
    y: object
    w: object
    row_offsets: np.ndarray
    x_offsets: np.ndarray
    dims: np.ndarray
    kinds: np.ndarray
    ridge: np.ndarray
    max_features: int
    max_dim: int

    @property
    def count(self) -> int:
        return int(self.dims.shape[0])

    @property
    def n_rows(self) -> int:
        return int(self.row_offsets[-1])

    def subset(self, idx):
        """Copy of systems `idx` (host numpy), same values."""

        idx = np.asarray(idx)
        xs, ys, ws, ro, xo = [], [], [], [0], [0]
        x = _host(self.x)
        y = _host(self.y)
        w = _host(self.w)
        for k in idx:
            r0, r1 = int(self.row_offsets[k]), int(self.row_offsets[k + 1])
            d = int(self.dims[k])
            x0 = int(self.x_offsets[k])
            xs.append(x[x0: x0 + (r1 - r0) * d])
            ys.append(y[r0:r1])
            ws.append(w[r0:r1])
            ro.append(ro[-1] + r1 - r0)
            xo.append(xo[-1] + (r1 - r0) * d)
        return RidgeWorkload(np.concatenate(xs), np.concatenate(ys), np.concatenate(ws),
                             np.array(ro, np.int64), np.array(xo[:-1], np.int64),
                             self.dims[idx].copy(), self.kinds[idx].copy(), self.ridge[idx].copy(),
                             self.max_features, self.max_dim)


def _host(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def ridge_systems(count: int = 65536, seed: int = 2, n_min: int = 64, n_max: int = 8192,
                  classes=RIDGE_CLASSES, device: str | None = None, only=None) -> RidgeWorkload:
    """Generate the batched ridge workload.

    Per-system parameters (n, d, features, ridge, weight halfspaces, target
    coefficients) come from numpy's PCG64 (seed) and do not depend on
    ``device``.  Rows are drawn on ``device`` ('cuda' -> torch's Philox
    generator, so the full ~110M-row set is generated in device memory) or,
    with ``device=None``, by numpy from a per-system seed; ``only`` then
    restricts generation to the listed systems (in that order).
    """

    rng = np.random.default_rng(seed)
    K = int(count)
    cls = np.arange(K) % len(classes)
    rng.shuffle(cls)
    dims = np.array([classes[c][0] for c in cls], dtype=np.int32)
    kinds = np.array([classes[c][1] for c in cls], dtype=np.int32)
    n = np.floor(np.exp(rng.uniform(np.log(n_min), np.log(n_max), K))).astype(np.int64)
    ridge = np.exp(rng.uniform(np.log(1e-8), np.log(1e-2), K))
    row_offsets = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    x_offsets = np.concatenate([[0], np.cumsum(n * dims)])[:-1].astype(np.int64)
    dmax = int(dims.max())
    # sigmoid-product weights: J ~ U{1..8} halfspaces per system
    J = rng.integers(1, 9, K)
    A = rng.normal(size=(K, 8, dmax))
    A[:, :, :] *= (np.arange(dmax)[None, None, :] < dims[:, None, None])
    A /= np.linalg.norm(A, axis=2, keepdims=True)
    B = rng.uniform(-0.5, 0.5, (K, 8))
    T = rng.uniform(0.05, 0.5, (K, 8))
    active = np.arange(8)[None, :] < J[:, None]
    # random quadratic target: coefficients N(0,1) on [1, x, x_i x_j]
    pq = 1 + dmax + dmax * (dmax + 1) // 2
    Q = rng.normal(size=(K, pq))
    gen_seed = int(rng.integers(0, 2**62))
    if device is None:
        idx = np.arange(K) if only is None else np.asarray(only, dtype=np.int64)
        out = _rows_numpy(idx, n, dims, kinds, ridge, A, B, T, active, Q, gen_seed, classes)
        out._full_meta = (row_offsets, dims, kinds)
        return out
    return _rows_torch(K, n, dims, kinds, ridge, row_offsets, x_offsets, A, B, T, active, Q,
                       gen_seed, classes, device)


def _quad_features(X, d):
    from itertools import combinations_with_replacement

    cols = [np.ones(X.shape[0])] + [X[:, i] for i in range(d)]
    cols += [X[:, i] * X[:, j] for i, j in combinations_with_replacement(range(d), 2)]
    return np.stack(cols, 1)


def _rows_numpy(idx, n, dims, kinds, ridge, A, B, T, active, Q, seed, classes):
    xs, ys, ws = [], [], []
    for k in idx:
        rng = np.random.default_rng([seed, int(k)])
        d = int(dims[k])
        X = rng.uniform(-1.0, 1.0, (int(n[k]), d))
        s = (X @ A[k, :, :d].T - B[k]) / T[k]
        sig = 1.0 / (1.0 + np.exp(-np.clip(s, -50, 50)))
        w = np.prod(np.where(active[k][None, :], sig, 1.0), axis=1)
        phi = _quad_features(X, d)
        y = phi @ Q[k, : phi.shape[1]] + rng.normal(0.0, 0.01, X.shape[0])
        xs.append(X.reshape(-1))
        ys.append(y)
        ws.append(w)
    pmax = max(kind_feature_count(d, kd) for d, kd in classes)
    nn = n[idx]
    ro = np.concatenate([[0], np.cumsum(nn)]).astype(np.int64)
    xo = np.concatenate([[0], np.cumsum(nn * dims[idx])])[:-1].astype(np.int64)
    return RidgeWorkload(np.concatenate(xs) if xs else np.zeros(0), np.concatenate(ys) if ys else np.zeros(0),
                         np.concatenate(ws) if ws else np.zeros(0), ro, xo, dims[idx].copy(),
                         kinds[idx].copy(), ridge[idx].copy(), pmax,
                         int(dims.max()) if len(dims) else 1)


def _rows_torch(K, n, dims, kinds, ridge, ro, xo, A, B, T, active, Q, seed, classes, device):
    import torch

    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    total = int(ro[-1])
    xtot = int((n * dims).sum())
    x = torch.empty(xtot, dtype=torch.float64, device=dev)
    y = torch.empty(total, dtype=torch.float64, device=dev)
    w = torch.empty(total, dtype=torch.float64, device=dev)
    At = torch.from_numpy(A).to(dev)
    Bt = torch.from_numpy(B).to(dev)
    Tt = torch.from_numpy(T).to(dev)
    act = torch.from_numpy(active).to(dev)
    Qt = torch.from_numpy(Q).to(dev)
    # process systems of equal d together in chunks of ~1M rows
    for dval in sorted(set(int(v) for v in dims)):
        ids = np.flatnonzero(dims == dval)
        iu, ju = np.triu_indices(dval)
        start = 0
        while start < ids.size:
            stop = start
            rows = 0
            while stop < ids.size and (rows < (1 << 20) or stop == start):
                rows += int(n[ids[stop]])
                stop += 1
            chunk = ids[start:stop]
            nn = torch.from_numpy(n[chunk]).to(dev)
            sys_of_row = torch.repeat_interleave(torch.arange(chunk.size, device=dev), nn)
            X = torch.rand((rows, dval), generator=g, device=dev, dtype=torch.float64) * 2.0 - 1.0
            kk = torch.from_numpy(chunk).to(dev)[sys_of_row]
            s = (torch.einsum("rd,rjd->rj", X, At[kk, :, :dval]) - Bt[kk]) / Tt[kk]
            sig = torch.sigmoid(torch.clamp(s, -50, 50))
            wv = torch.where(act[kk], sig, torch.ones_like(sig)).prod(dim=1)
            quad = X[:, iu] * X[:, ju]
            phi = torch.cat([torch.ones((rows, 1), device=dev, dtype=torch.float64), X, quad], 1)
            yv = (phi * Qt[kk, : phi.shape[1]]).sum(1)
            yv += 0.01 * torch.randn(rows, generator=g, device=dev, dtype=torch.float64)
            # scatter to the segmented layout
            rstart = torch.from_numpy(ro[chunk]).to(dev)
            local = torch.arange(rows, device=dev) - torch.repeat_interleave(
                torch.cumsum(nn, 0) - nn, nn)
            dst = rstart[sys_of_row] + local
            y[dst] = yv
            w[dst] = wv
            xstart = torch.from_numpy(xo[chunk]).to(dev)
            xdst = (xstart[sys_of_row] + local * dval)[:, None] + torch.arange(dval, device=dev)[None, :]
            x[xdst.reshape(-1)] = X.reshape(-1)
            del X, s, sig, wv, quad, phi, yv, dst, xdst
            start = stop
    pmax = max(kind_feature_count(d, kd) for d, kd in classes)
    return RidgeWorkload(x, y, w, ro, xo, dims, kinds, ridge, pmax, int(dims.max()))


def ridge_meta(wl: RidgeWorkload):
    """(row_offsets, dims, kinds) of the full mix a (possibly row-less) workload was drawn from."""

    return wl._full_meta


@dataclass
class SplitWorkload:
    """Node-sorted split-search inputs: x (sum n_k * d,), y (sum n_k,), CSR offsets."""

    x: object
    y: object
    row_offsets: np.ndarray
    dims: np.ndarray
    kinds: np.ndarray
    theta0: object  # (K, R, d + 1) restart normals and thresholds
    temperature: np.ndarray
    ridge: np.ndarray
    d: int

    @property
    def count(self) -> int:
        return int(self.dims.size)

    @property
    def n_rows(self) -> int:
        return int(self.row_offsets[-1])


def split_nodes(count: int = 4096, seed: int = 3, d: int = 16, n_min: int = 256, n_max: int = 16384,
                restarts: int = 16, temperature: float = 0.2, ridge: float = 1e-6,
                device: str = "cuda") -> SplitWorkload:
    """Batched split-search nodes: each node a random axis box inside [-1,1]^d
    (side lengths U[0.25, 1] * 2), x uniform in the box, y = 8 Gaussian bumps
    (widths U(0.1, 0.6), amplitudes N(0,1)) + a linear trend with N(0,1)
    coefficients; R restart normals per node (unit Gaussian w, z = the median
    of x.w over the node).  Node parameters come from numpy's PCG64 (seed);
    rows are drawn on ``device`` by torch's Philox generator."""

    import torch

    rng = np.random.default_rng(seed)
    K = int(count)
    n = np.floor(np.exp(rng.uniform(np.log(n_min), np.log(n_max), K))).astype(np.int64)
    side = rng.uniform(0.25, 1.0, (K, d)) * 2.0
    lo = rng.uniform(-1.0, 1.0 - side)
    centres = rng.uniform(-1.0, 1.0, (8, d))
    widths = rng.uniform(0.1, 0.6, 8)
    amps = rng.normal(size=8)
    trend = rng.normal(size=d)
    W0 = rng.normal(size=(K, restarts, d))
    W0 /= np.linalg.norm(W0, axis=2, keepdims=True)
    gen_seed = int(rng.integers(0, 2**62))
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(gen_seed)
    ro = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
    total = int(ro[-1])
    nt = torch.from_numpy(n).to(dev)
    node = torch.repeat_interleave(torch.arange(K, device=dev), nt)
    lo_t = torch.from_numpy(lo).to(dev)
    side_t = torch.from_numpy(side).to(dev)
    x = torch.empty((total, d), dtype=torch.float64, device=dev)
    y = torch.empty(total, dtype=torch.float64, device=dev)
    C_t = torch.from_numpy(centres).to(dev)
    Wd = torch.from_numpy(widths).to(dev)
    Am = torch.from_numpy(amps).to(dev)
    Tr = torch.from_numpy(trend).to(dev)
    step = 1 << 21
    for s in range(0, total, step):
        e = min(total, s + step)
        kk = node[s:e]
        X = lo_t[kk] + side_t[kk] * torch.rand((e - s, d), generator=g, device=dev, dtype=torch.float64)
        r2 = ((X[:, None, :] - C_t[None]) ** 2).sum(-1)
        y[s:e] = (Am * torch.exp(-r2 / (2.0 * Wd ** 2))).sum(1) + X @ Tr
        x[s:e] = X
    theta0 = torch.empty((K, restarts, d + 1), dtype=torch.float64, device=dev)
    W0_t = torch.from_numpy(W0).to(dev)
    theta0[:, :, :d] = W0_t
    for k0 in range(0, K, 256):
        k1 = min(K, k0 + 256)
        r0, r1 = int(ro[k0]), int(ro[k1])
        proj = torch.einsum("nd,nrd->nr", x[r0:r1], W0_t[node[r0:r1]])
        for k in range(k0, k1):
            a, b = int(ro[k]) - r0, int(ro[k + 1]) - r0
            theta0[k, :, d] = proj[a:b].median(dim=0).values if b > a else 0.0
    return SplitWorkload(x.reshape(-1), y, ro, np.full(K, d, np.int32), np.full(K, N.FEATURES_AFFINE, np.int32),
                         theta0, np.full(K, temperature), np.full(K, ridge), d)


@dataclass
class PolytopeWorkload:
    """Chains in per-chain polytopes [-1,1]^d cut by k oblique halfspaces."""

    lo: object
    hi: object
    row_offsets: object
    A: object
    b: object
    max_rows: int
    x0: object
    chain_polytope: object
    seeds: object
    d: int


def polytopes(count: int = 16384, d: int = 8, seed: int = 4, k_min: int = 4, k_max: int = 12,
              device: str = "cuda") -> PolytopeWorkload:
    """One polytope per chain: box [-1,1]^d and k ~ U{k_min..k_max} unit
    halfspaces a.x <= b with b = a.c + r, c ~ U[-0.5,0.5]^d, r ~ U[0.05, 0.5],
    so a ball of radius >= 0.05 around the start c is feasible."""

    import torch

    rng = np.random.default_rng([seed, d])
    Cn = int(count)
    k = rng.integers(k_min, k_max + 1, Cn)
    c = rng.uniform(-0.5, 0.5, (Cn, d))
    ro = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    A = rng.normal(size=(int(ro[-1]), d))
    A /= np.linalg.norm(A, axis=1, keepdims=True)
    owner = np.repeat(np.arange(Cn), k)
    r = rng.uniform(0.05, 0.5, owner.size)
    b = np.einsum("ij,ij->i", A, c[owner]) + r
    dev = torch.device(device)
    to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)
    return PolytopeWorkload(to(np.full((Cn, d), -1.0), torch.float64), to(np.full((Cn, d), 1.0), torch.float64),
                            to(ro, torch.int64), to(A, torch.float64), to(b, torch.float64), int(k_max),
                            to(c, torch.float64), to(np.arange(Cn), torch.int32),
                            to((np.uint64(seed) << np.uint64(32)) + np.arange(Cn, dtype=np.uint64), torch.int64), d)


def bumps_ridge_2d(seed: int = 1):
    """Target on [-1,1]^2: 3 Gaussian bumps (centres U[-0.8,0.8]^2, widths
    U[0.2,0.5], amplitudes N(0,1)) + tanh(8 (a.x - b)), a a random unit
    vector, b ~ U(-0.3, 0.3).  Returns a vectorised numpy callable."""

    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.8, 0.8, (3, 2))
    widths = rng.uniform(0.2, 0.5, 3)
    amps = rng.normal(size=3)
    a = rng.normal(size=2)
    a /= np.linalg.norm(a)
    b = rng.uniform(-0.3, 0.3)

    def f(X):
        X = np.atleast_2d(X)
        r2 = ((X[:, None, :] - centres[None]) ** 2).sum(-1)
        return (amps * np.exp(-r2 / (2 * widths ** 2))).sum(1) + np.tanh(8 * (X @ a - b))

    return f


def random_tree(depth: int = 8, d: int = 4, seed: int = 6):
    """A full regression tree of the given depth on [-1,1]^d for prediction
    benchmarks: random unit split normals with thresholds in (-0.2, 0.2),
    affine leaves with N(0,1) coefficients."""

    from .models import AffineRidgeModel
    from .tree import LeafNode, RegressionTree, SplitNode

    rng = np.random.default_rng(seed)

    def grow(level, node_id):
        if level == depth:
            m = AffineRidgeModel()
            m.coef_ = rng.normal(size=d + 1)
            return LeafNode(m, depth=level, node_id=node_id)
        w = rng.normal(size=d)
        w /= np.linalg.norm(w)
        return SplitNode(w, float(rng.uniform(-0.2, 0.2)), grow(level + 1, node_id + "/L"),
                         grow(level + 1, node_id + "/R"), depth=level, node_id=node_id)

    return RegressionTree(grow(0, "root"))
