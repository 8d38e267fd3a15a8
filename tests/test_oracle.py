"""The CPU oracle reproduces the reference's own outputs (golden fixtures made from it)."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import ridge as O


def load_ridge_cases():
    g = np.load(GOLDEN / "ridge_golden.npz")
    for i in range(int(g["count"])):
        kind, lam, solver = g[f"c{i}_meta"]
        yield dict(X=g[f"c{i}_X"], y=g[f"c{i}_y"], w=g[f"c{i}_w"], kind=int(kind), ridge=float(lam),
                   solver=("normal", "auto", "qr", "svd")[int(solver)], beta=g[f"c{i}_beta"],
                   ridge_eff=float(g[f"c{i}_ridge_eff"]), solver_used=str(g[f"c{i}_solver_used"]),
                   cond=float(g[f"c{i}_cond"]), rank=int(g[f"c{i}_rank"]))


@pytest.mark.parametrize("case", list(load_ridge_cases()), ids=lambda c: f"{c['solver']}-k{c['kind']}-n{len(c['y'])}")
def test_ridge_oracle_matches_reference(case):
    phi = O.features(case["X"], case["kind"])
    res = O.solve_weighted_ridge(phi, case["y"], case["w"], case["ridge"], solver=case["solver"])
    np.testing.assert_allclose(res["coefficients"], case["beta"], rtol=1e-12, atol=1e-12)
    assert res["ridge_effective"] == pytest.approx(case["ridge_eff"], rel=1e-14)
    assert res["solver_used"] == case["solver_used"]
    if case["solver_used"] == "svd":
        assert res["rank"] == case["rank"]
        np.testing.assert_allclose(res["cond_estimate"], case["cond"], rtol=1e-12)


def test_golden_set_covers_fallback_and_kinds():
    cases = list(load_ridge_cases())
    assert any(c["solver_used"] == "qr" for c in cases)
    assert any(c["solver_used"] == "svd" and c["rank"] < len(c["beta"]) for c in cases)
    assert {c["kind"] for c in cases} == {0, 1, 2, 3, 4}


def test_feature_order_matches_sklearn():
    from sklearn.preprocessing import PolynomialFeatures

    X = np.random.default_rng(3).normal(size=(7, 5))
    np.testing.assert_array_equal(O.features(X, O.POLY2), PolynomialFeatures(2).fit_transform(X))
    np.testing.assert_array_equal(O.features(X, O.POLY2_NOBIAS),
                                  PolynomialFeatures(2, include_bias=False).fit_transform(X))
    np.testing.assert_array_equal(O.features(X, O.AFFINE), np.hstack([X, np.ones((7, 1))]))
