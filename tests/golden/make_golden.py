"""Generate golden fixtures from the reference implementation itself.

Run in a container that has the reference source tree:

    python tests/golden/make_golden.py /path/to/reference

The reference package is imported under the name ``art_ref`` (it is also
called ``art``), its outputs on small seeded inputs are written to
``tests/golden/*.npz``, and the oracle restatement is checked against them
before anything is written.  The GPU box never needs the reference: tests
read only the committed fixtures.
"""

from __future__ import annotations

import importlib.util
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))


def import_reference(root: Path):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/art_ref_numba_cache")
    spec = importlib.util.spec_from_file_location(
        "art_ref", root / "art" / "__init__.py", submodule_search_locations=[str(root / "art")]
    )
    mod = importlib.util.module_from_spec(spec)
    sys.modules["art_ref"] = mod
    spec.loader.exec_module(mod)
    return mod


def ridge_cases(ref):
    """Weighted ridge systems covering kinds, solvers, weights, fallbacks."""

    from oracle import ridge as O

    rng = np.random.default_rng(20240601)
    cases = []
    # (n, d, kind, ridge, solver, weighted)
    specs = [
        (40, 2, O.AFFINE, 1e-6, "normal", True),
        (97, 3, O.POLY2, 1e-8, "normal", True),
        (257, 8, O.AFFINE, 1e-4, "normal", True),
        (300, 8, O.POLY2, 1e-3, "normal", True),
        (520, 16, O.POLY2, 1e-2, "normal", True),
        (64, 5, O.POLY1, 0.0, "normal", False),
        (31, 4, O.POLY2_NOBIAS, 1e-5, "normal", True),
        (33, 6, O.POLY1_NOBIAS, 1e-7, "auto", True),
        (200, 16, O.AFFINE, 1e-8, "auto", True),
        (150, 4, O.POLY2, 1e-6, "auto", True),
        (1, 2, O.AFFINE, 1e-3, "normal", False),
    ]
    for n, d, kind, lam, solver, weighted in specs:
        X = rng.uniform(-1, 1, (n, d))
        y = np.sin(3 * X[:, 0]) + X[:, -1] ** 2 + 0.01 * rng.normal(size=n)
        w = rng.uniform(0.0, 1.0, n) ** 2 if weighted else np.ones(n)
        cases.append((X, y, w, kind, lam, solver))
    # ill-conditioned design from the reference's own auto->QR test (test_models.py:120-142)
    base = rng.normal(size=120)
    X = np.column_stack([base, base + 1e-7 * rng.normal(size=120), rng.normal(size=120)])
    cases.append((X, rng.normal(size=120), np.ones(120), O.POLY1_NOBIAS, 0.0, "auto"))
    # direct least-squares solvers (gelsy / gelsd on the augmented system),
    # drawn from their own stream so the cases above keep their inputs
    rng2 = np.random.default_rng(20240602)
    for n, d, kind, lam, solver, weighted in [
        (90, 3, O.AFFINE, 1e-6, "qr", True),
        (120, 4, O.POLY2, 1e-5, "svd", True),
        (400, 8, O.POLY2, 1e-3, "svd", True),
        (60, 2, O.AFFINE, 0.0, "svd", False),
        (300, 16, O.AFFINE, 1e-8, "svd", True),
    ]:
        X = rng2.uniform(-1, 1, (n, d))
        y = np.sin(3 * X[:, 0]) + X[:, -1] ** 2 + 0.01 * rng2.normal(size=n)
        w = rng2.uniform(0.0, 1.0, n) ** 2 if weighted else np.ones(n)
        cases.append((X, y, w, kind, lam, solver))
    # rank-deficient design without ridge: gelsd's minimum-norm solution
    base = rng2.uniform(-1, 1, (80, 2))
    X = np.column_stack([base, base[:, 0] + base[:, 1]])
    cases.append((X, rng2.normal(size=80), np.ones(80), O.POLY1_NOBIAS, 0.0, "svd"))
    out = {}
    for i, (X, y, w, kind, lam, solver) in enumerate(cases):
        phi = O.features(X, kind)
        res = ref.models.solve_weighted_ridge(phi, y, w, lam, solver=solver)
        mine = O.solve_weighted_ridge(phi, y, w, lam, solver=solver)
        np.testing.assert_allclose(mine["coefficients"], res.coefficients, rtol=1e-12, atol=1e-12)
        assert mine["solver_used"] == res.solver_used
        # sklearn basis equals the oracle's feature order
        if kind in (O.POLY2, O.POLY1, O.POLY2_NOBIAS, O.POLY1_NOBIAS):
            deg = 2 if kind in (O.POLY2, O.POLY2_NOBIAS) else 1
            bias = kind in (O.POLY1, O.POLY2)
            pm = ref.models.PolynomialRidgeModel(degree=deg, include_bias=bias)
            np.testing.assert_array_equal(pm.prepare_design(X).matrix, phi)
        else:
            np.testing.assert_array_equal(ref.models.augment_features(X), phi)
        out[f"c{i}_X"] = X
        out[f"c{i}_y"] = y
        out[f"c{i}_w"] = w
        out[f"c{i}_meta"] = np.array([kind, lam, {"normal": 0, "auto": 1, "qr": 2, "svd": 3}[solver]], dtype=float)
        out[f"c{i}_rank"] = np.array(-1 if res.rank is None else int(res.rank))
        out[f"c{i}_beta"] = res.coefficients
        out[f"c{i}_ridge_eff"] = np.array(res.ridge_effective)
        out[f"c{i}_solver_used"] = np.array(res.solver_used)
        out[f"c{i}_cond"] = np.array(np.nan if res.cond_estimate is None else res.cond_estimate)
    out["count"] = np.array(len(cases))
    np.savez_compressed(HERE / "ridge_golden.npz", **out)
    print("ridge cases:", len(cases))


SPLIT_SPECS = [
    # (seed, n, d, kind, T, ridge, restarts, max_iters, extra splitter kwargs)
    (101, 200, 2, 0, 0.1, 1e-6, 1, 30, {}),
    (102, 150, 3, 2, 0.3, 1e-4, 2, 15, {}),
    (103, 300, 4, 0, 0.05, 1e-6, 3, 40, {"adaptive_alpha": False, "alpha0": 0.5}),
    (104, 120, 2, 0, 0.02, 1e-6, 1, 25, {"min_side_points": 40, "min_side_fallback": True,
                                         "min_side_fraction": 0.0}),
    (105, 400, 6, 0, 0.2, 1e-5, 2, 20, {"max_backtracks": 6, "heavy_backtrack_threshold": 3}),
    (106, 250, 3, 1, 0.15, 1e-3, 1, 12, {"alpha_max": 1e8, "max_line_search_failures": 5}),
]


def split_target(X, rng):
    a = rng.normal(size=X.shape[1])
    a /= np.linalg.norm(a)
    return np.tanh(6 * (X @ a - 0.1)) + 0.3 * X[:, 0] ** 2 + 0.01 * rng.normal(size=X.shape[0])


def split_cases(ref):
    from oracle import ridge as O
    from oracle import split as S

    out = {}
    for i, (seed, n, d, kind, T, lam, R, iters, extra) in enumerate(SPLIT_SPECS):
        rng = np.random.default_rng(seed)
        X = rng.uniform(-1, 1, (n, d))
        y = split_target(X, rng)
        if kind == O.AFFINE:
            model = ref.models.AffineRidgeModel(ridge=lam)
        else:
            model = ref.models.PolynomialRidgeModel(degree=2 if kind == O.POLY2 else 1, ridge=lam)
        kw = dict(max_iters=iters, n_restarts=R, random_state=seed + 1000)
        kw.update(extra)
        splitter = ref.splitters.SoftObliqueSplitter(model, T, **kw)
        res = splitter.split(X, y)
        # oracle with the same theta0 draws
        init_rng = np.random.default_rng(seed + 1000)
        theta0s = [S.initialize_theta(X, init_rng) for _ in range(R)]
        params = S.Params(max_iters=iters, n_restarts=R, **{k: v for k, v in extra.items()})
        phi = O.features(X, kind)
        parent = O.solve_weighted_ridge(phi, y, np.ones(n), lam)["coefficients"]
        parent_loss = float(np.mean((y - phi @ parent) ** 2))
        mine = S.split(X, y, theta0s, T, kind, lam, parent_loss, params)
        np.testing.assert_allclose(np.r_[mine["w"], mine["z"]], np.r_[res.w, res.z], rtol=1e-9, atol=1e-11)
        assert mine["stop_reason"] == res.stop_reason and mine["n_iters"] == res.n_iters
        np.testing.assert_allclose(mine["losses"], res.metadata["soft_loss_history"], rtol=1e-9, atol=1e-13)
        np.testing.assert_allclose(mine["loss"], res.loss, rtol=1e-9)
        assert mine["n_right"] == res.n_right
        out[f"s{i}_X"] = X
        out[f"s{i}_y"] = y
        out[f"s{i}_theta0"] = np.array(theta0s)
        out[f"s{i}_meta"] = np.array([kind, T, lam, R, iters, parent_loss], dtype=float)
        out[f"s{i}_extra"] = np.array(repr(extra))
        out[f"s{i}_theta"] = np.r_[res.w, res.z]
        out[f"s{i}_loss"] = np.array(res.loss)
        out[f"s{i}_n_right"] = np.array(res.n_right)
        out[f"s{i}_n_iters"] = np.array(res.n_iters)
        out[f"s{i}_stop"] = np.array(res.stop_reason)
        out[f"s{i}_soft_losses"] = np.array(res.metadata["soft_loss_history"])
        out[f"s{i}_steps"] = np.array(res.metadata["step_size_history"])
        out[f"s{i}_backtracks"] = np.array(res.metadata["backtrack_history"])
        out[f"s{i}_grad_norms"] = np.array(res.metadata["projected_grad_norm_history"])
        out[f"s{i}_beta_left"] = res.left_model.coef_
        out[f"s{i}_beta_right"] = res.right_model.coef_
        out[f"s{i}_fallback"] = np.array(bool(res.metadata.get("min_side_fallback", False)))
    out["count"] = np.array(len(SPLIT_SPECS))
    np.savez_compressed(HERE / "split_golden.npz", **out)
    print("split cases:", len(SPLIT_SPECS))


def har_polytope(rng, d, k):
    """Box [-1,1]^d cut by k halfspaces a.x <= a.c + r with a Chebyshev ball at c."""
    c = rng.uniform(-0.5, 0.5, d)
    A = rng.normal(size=(k, d))
    A /= np.linalg.norm(A, axis=1, keepdims=True)
    r = rng.uniform(0.05, 0.5, k)
    return A, A @ c + r, c


class FixedStream:
    """Serves injected draws through the Generator calls HitAndRunSampler makes."""

    def __init__(self, directions, uniforms):
        self.directions, self.uniforms = directions, uniforms
        self.i = self.j = 0

    def normal(self, size):
        v = self.directions[self.i].copy()
        self.i += 1
        return v

    def uniform(self, low, high):
        v = self.uniforms[self.j]
        self.j += 1
        return float(low + v * (high - low))


def har_cases(ref):
    import importlib

    from oracle import sampling as H

    numba_sampling = importlib.import_module("art_ref._numba_sampling")
    out = {}
    # numba batched form, chain-major injected draws
    specs = [(201, 2, 3, 16, 5, 2, 7), (202, 8, 6, 12, 3, 4, 9), (203, 16, 10, 8, 0, 5, 6),
             (204, 32, 12, 4, 2, 3, 5)]
    for i, (seed, d, k, C, burn, thin, rounds) in enumerate(specs):
        rng = np.random.default_rng(seed)
        Ao, bo, c = har_polytope(rng, d, k)
        Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
        A = np.vstack([Ab, Ao])
        b = np.concatenate([bb, bo])
        steps = burn + thin * rounds
        x0 = np.repeat(c[None, :], C, axis=0) + 0.01 * rng.uniform(-1, 1, (C, d))
        dirs = rng.normal(size=(C, steps, d))
        unif = rng.random(size=(C, steps))
        pts = x0.copy()
        slack = b[None, :] - pts @ A.T
        cp = (dirs.reshape(-1, d) @ np.ascontiguousarray(A.T)).reshape(C, steps, -1)
        samples = np.empty((rounds * C, d))
        numba_sampling.sample_precomputed_chains_parallel(pts, slack, dirs, cp, unif, burn, thin, samples)
        mine, last = H.chains_batched(A, b, x0, dirs, unif, burn, thin, rounds)
        np.testing.assert_allclose(mine.reshape(-1, d), samples, rtol=1e-13, atol=1e-13)
        out[f"b{i}_meta"] = np.array([d, k, C, burn, thin, rounds])
        out[f"b{i}_Ao"], out[f"b{i}_bo"], out[f"b{i}_x0"] = Ao, bo, x0
        out[f"b{i}_dirs"], out[f"b{i}_unif"] = dirs, unif
        out[f"b{i}_samples"] = samples.reshape(rounds, C, d)
    # scalar HitAndRunSampler with injected draws
    sspecs = [(301, 2, 2, 3, 2, 12), (302, 5, 4, 0, 4, 10), (303, 12, 8, 6, 3, 8)]
    for i, (seed, d, k, burn, thin, n) in enumerate(sspecs):
        rng = np.random.default_rng(seed)
        Ao, bo, c = har_polytope(rng, d, k)
        Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
        A = np.vstack([Ab, Ao])
        b = np.concatenate([bb, bo])
        region = ref.domain.PolytopeRegion(A, b)
        steps = burn + thin * n
        dirs = rng.normal(size=(steps, d))
        unif = rng.random(size=steps)
        stream = FixedStream(dirs, unif)
        old = ref.sampling.as_rng
        ref.sampling.as_rng = lambda _: stream
        try:
            samples = ref.sampling.HitAndRunSampler(burn_in=burn, thinning=thin).sample(region, n, x0=c)
        finally:
            ref.sampling.as_rng = old
        mine = H.chain_scalar(A, b, c, dirs, unif, burn, thin, n)
        np.testing.assert_allclose(mine, samples, rtol=1e-13, atol=1e-13)
        out[f"s{i}_meta"] = np.array([d, k, burn, thin, n])
        out[f"s{i}_Ao"], out[f"s{i}_bo"], out[f"s{i}_x0"] = Ao, bo, c
        out[f"s{i}_dirs"], out[f"s{i}_unif"] = dirs, unif
        out[f"s{i}_samples"] = samples
    # autocorrelation estimator
    series = np.cumsum(np.random.default_rng(7).normal(size=(300, 3)), axis=0)
    lags = (1, 2, 5, 10, 50)
    acf = ref.sampling.autocorrelation_by_lag(series, lags)
    np.testing.assert_allclose(H.autocorrelation_by_lag(series, lags), acf, rtol=1e-13, atol=1e-13)
    out["acf_series"], out["acf_lags"], out["acf"] = series, np.array(lags), acf
    out["batched_count"] = np.array(len(specs))
    out["scalar_count"] = np.array(len(sspecs))
    np.savez_compressed(HERE / "har_golden.npz", **out)
    print("har cases:", len(specs), len(sspecs))


SAMPLER_SPECS = [
    # (seed, class, d, k oblique rows, n, kwargs, x0 kind: none / point / pool, spectrum)
    (501, "BatchedHitAndRunSampler", 3, 2, 30, dict(burn_in=5, thinning=3, n_chains=7), "pool", False),
    (502, "NumbaBatchedHitAndRunSampler", 5, 4, 23, dict(burn_in=0, thinning=2, n_chains=5), "pool", False),
    (503, "ParallelNumbaBatchedHitAndRunSampler", 4, 3, 40,
     dict(burn_in=4, thinning=2, n_chains=9, random_threads=4), "point", False),
    (504, "ParallelNumbaBatchedHitAndRunSampler", 3, 2, 17,
     dict(burn_in=2, thinning=1, n_chains=6, parallel_random=False), "pool", True),
    (505, "BatchedHitAndRunSampler", 2, 1, 12, dict(burn_in=3, thinning=0, n_chains=4), "none", True),
]


def sampler_cases(ref):
    """The reference's batched sampler classes end to end (their own draws)."""

    from oracle import sampling as H

    out = {}
    for i, (seed, cls, d, k, n, kw, x0kind, spectrum) in enumerate(SAMPLER_SPECS):
        rng = np.random.default_rng(seed)
        Ao, bo, c = har_polytope(rng, d, k)
        Ab, bb = H.box_rows(-np.ones(d), np.ones(d))
        A, b = np.vstack([Ab, Ao]), np.concatenate([bb, bo])
        region = ref.domain.PolytopeRegion(A, b)
        if x0kind == "pool":
            pool = c[None, :] + 0.02 * rng.uniform(-1, 1, (5, d))
        elif x0kind == "point":
            pool = c[None, :].copy()
        else:
            pool = np.zeros((0, d))
        extra = dict(kw)
        if spectrum:
            Q, _ = np.linalg.qr(rng.normal(size=(d, d)))
            extra.update(direction_eigenvectors=Q, direction_eigenvalues=rng.uniform(0.1, 2.0, d))
        sampler = getattr(ref.sampling, cls)(**extra)
        x0 = None if x0kind == "none" else (pool[0] if x0kind == "point" else pool)
        samples = sampler.sample(region, n, random_state=seed + 7, x0=x0)
        out[f"m{i}_A"], out[f"m{i}_b"], out[f"m{i}_pool"] = A, b, pool
        out[f"m{i}_spec"] = np.array(repr((seed, cls, d, k, n, kw, x0kind)))
        if spectrum:
            out[f"m{i}_vecs"] = extra["direction_eigenvectors"]
            out[f"m{i}_vals"] = extra["direction_eigenvalues"]
        out[f"m{i}_samples"] = samples
    out["count"] = np.array(len(SAMPLER_SPECS))
    np.savez_compressed(HERE / "har_sampler_golden.npz", **out)
    print("sampler cases:", len(SAMPLER_SPECS))


def c1_target(seed):
    """Sum of 3 Gaussian bumps + tanh ridge (the C1 target family)."""
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

    return f, (centres, widths, amps, a, b)


def flatten_tree(ref, tree):
    rows = []
    for node in tree.iter_nodes():
        if isinstance(node, ref.tree.SplitNode):
            rows.append((node.node_id, node.status, np.r_[node.w, node.z], None,
                         node.metadata.get("n_samples")))
        else:
            rows.append((node.node_id, node.status, None, np.asarray(node.model.coef_),
                         node.metadata.get("n_samples")))
    return rows


TREE_SPECS = [
    # (seed, traversal, sample_count, max_depth, isotropic, threshold, restarts)
    (401, "dfs", 200, 3, False, 0.02, 1),
    (402, "bfs", 160, 3, True, 0.02, 1),
    (403, "dfs", 120, 2, True, 0.05, 2),
]


def tree_cases(ref):
    out = {}
    for i, (seed, trav, count, depth, iso, thr, R) in enumerate(TREE_SPECS):
        f, params = c1_target(seed)
        model = ref.models.AffineRidgeModel(ridge=1e-6, solver="normal")
        splitter = ref.splitters.SoftObliqueSplitter(model, 0.05, max_iters=40, n_restarts=R, min_side_points=8,
                                                     min_side_fraction=0.0)
        builder = ref.builder.RegressionTreeBuilder(
            domain=ref.domain.BoxDomain.hypercube(2, -1.0, 1.0), oracle=f, model_template=model,
            splitter=splitter, error_threshold=thr, max_depth=depth, sample_count=count,
            isotropic_sampling=iso, temperature_config=ref.temperature.TemperatureConfig(strategy="splitter"),
            random_state=seed, oracle_vectorized=True, traversal=trav,
            sampler=ref.sampling.HitAndRunSampler(burn_in=0, thinning=5))
        res = builder.build()
        rows = flatten_tree(ref, res.tree)
        out[f"t{i}_ids"] = np.array([r[0] for r in rows])
        out[f"t{i}_status"] = np.array([r[1] for r in rows])
        out[f"t{i}_theta"] = np.array([r[2] if r[2] is not None else np.full(3, np.nan) for r in rows])
        out[f"t{i}_coef"] = np.array([r[3] if r[3] is not None else np.full(3, np.nan) for r in rows])
        out[f"t{i}_nsamples"] = np.array([-1 if r[4] is None else r[4] for r in rows])
        out[f"t{i}_queries"] = np.array(res.oracle_queries)
        out[f"t{i}_target"] = np.concatenate([np.ravel(p) for p in params[:4]] + [[params[4]]])
        Xt = np.random.default_rng(seed + 1).uniform(-1, 1, (500, 2))
        out[f"t{i}_Xtest"] = Xt
        out[f"t{i}_pred"] = res.tree.predict(Xt)
        print(f"tree {i}: {res.tree.num_nodes()} nodes, {res.oracle_queries} queries")
    out["count"] = np.array(len(TREE_SPECS))
    np.savez_compressed(HERE / "tree_golden.npz", **out)


def c1tree_cases(ref):
    """One build at the C1 configuration: d = 2, 4096 samples per node, depth
    <= 6, at least 32 points per side, T = 0.05 absolute, 100 iterations,
    affine ridge leaves with lambda = 1e-6 (DFS, the reference's default)."""

    seed = 411
    f, params = c1_target(seed)
    model = ref.models.AffineRidgeModel(ridge=1e-6, solver="normal")
    splitter = ref.splitters.SoftObliqueSplitter(model, 0.05, max_iters=100, n_restarts=1, min_side_points=32,
                                                 min_side_fraction=0.0)
    builder = ref.builder.RegressionTreeBuilder(
        domain=ref.domain.BoxDomain.hypercube(2, -1.0, 1.0), oracle=f, model_template=model,
        splitter=splitter, error_threshold=0.02, max_depth=6, sample_count=4096, isotropic_sampling=False,
        temperature_config=ref.temperature.TemperatureConfig(strategy="splitter"), random_state=seed,
        oracle_vectorized=True, traversal="dfs", sampler=ref.sampling.HitAndRunSampler(burn_in=0, thinning=5))
    res = builder.build()
    rows = flatten_tree(ref, res.tree)
    out = {
        "ids": np.array([r[0] for r in rows]),
        "status": np.array([r[1] for r in rows]),
        "theta": np.array([r[2] if r[2] is not None else np.full(3, np.nan) for r in rows]),
        "coef": np.array([r[3] if r[3] is not None else np.full(3, np.nan) for r in rows]),
        "nsamples": np.array([-1 if r[4] is None else r[4] for r in rows]),
        "queries": np.array(res.oracle_queries),
        "target": np.concatenate([np.ravel(p) for p in params[:4]] + [[params[4]]]),
        "seed": np.array(seed),
    }
    Xt = np.random.default_rng(seed + 1).uniform(-1, 1, (4000, 2))
    out["Xtest"] = Xt
    out["pred"] = res.tree.predict(Xt)
    out["ytest"] = f(Xt)
    np.savez_compressed(HERE / "tree_c1_golden.npz", **out)
    print(f"C1 tree: {res.tree.num_nodes()} nodes, {res.oracle_queries} queries")


def main():
    root = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ART_REFERENCE", ""))
    if not (root / "art" / "__init__.py").exists():
        raise SystemExit("usage: make_golden.py /path/to/reference (the tree holding art/)")
    ref = import_reference(root)
    which = sys.argv[2:] or ["ridge"]
    for name in which:
        globals()[f"{name}_cases"](ref)


if __name__ == "__main__":
    main()
