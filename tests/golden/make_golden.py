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
        out[f"c{i}_meta"] = np.array([kind, lam, {"normal": 0, "auto": 1}[solver]], dtype=float)
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
