"""The oracle's depth-first tree build reproduces the reference's trees
(fixtures made by the reference builder): node ids, statuses, oracle query
counts, split planes and leaf coefficients, and held-out predictions."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import builder as B
from oracle import ridge as O
from oracle import split as S


def target_from(params):
    centres = params[:6].reshape(3, 2)
    widths, amps, a, b = params[6:9], params[9:12], params[12:14], params[14]

    def f(X):
        X = np.atleast_2d(X)
        r2 = ((X[:, None, :] - centres[None]) ** 2).sum(-1)
        return (amps * np.exp(-r2 / (2 * widths ** 2))).sum(1) + np.tanh(8 * (X @ a - b))

    return f


def _check(root, ids, status, theta, coef, queries, got_queries):
    nodes = list(B.iter_nodes(root))
    assert [n.node_id for n in nodes] == list(ids)
    assert [n.status for n in nodes] == list(status)
    assert got_queries == int(queries)
    for n, th, cf in zip(nodes, theta, coef):
        if n.left is not None:
            np.testing.assert_allclose(np.r_[n.w, n.z], th, rtol=1e-9, atol=1e-11)
        else:
            np.testing.assert_allclose(n.coef, cf, rtol=1e-9, atol=1e-11)


def test_oracle_builder_reproduces_reference_dfs_tree():
    G = np.load(GOLDEN / "tree_golden.npz")
    b = B.Builder(-np.ones(2), np.ones(2), target_from(G["t0_target"]), O.AFFINE, 1e-6, 0.05, 0.02, 3, 200,
                  S.Params(max_iters=40, n_restarts=1, min_side_points=8, min_side_fraction=0.0),
                  burn_in=0, thinning=5, random_state=401)
    root = b.build()
    _check(root, G["t0_ids"], G["t0_status"], G["t0_theta"], G["t0_coef"], G["t0_queries"], b.queries)
    np.testing.assert_allclose(B.predict(root, G["t0_Xtest"], O.AFFINE), G["t0_pred"], rtol=1e-9, atol=1e-11)


def test_oracle_builder_reproduces_reference_c1_tree():
    G = np.load(GOLDEN / "tree_c1_golden.npz")
    b = B.Builder(-np.ones(2), np.ones(2), target_from(G["target"]), O.AFFINE, 1e-6, 0.05, 0.02, 6, 4096,
                  S.Params(max_iters=100, n_restarts=1, min_side_points=32, min_side_fraction=0.0),
                  burn_in=0, thinning=5, random_state=int(G["seed"]))
    root = b.build()
    _check(root, G["ids"], G["status"], G["theta"], G["coef"], G["queries"], b.queries)
    np.testing.assert_allclose(B.predict(root, G["Xtest"][:500], O.AFFINE), G["pred"][:500], rtol=1e-9,
                               atol=1e-11)
