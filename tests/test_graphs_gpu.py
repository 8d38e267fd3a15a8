"""Captured split levels replay exactly what the eager launch sequence computes."""

import numpy as np
import pytest

from conftest import gpu_available
from oracle import ridge as O

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

FIELDS = ("theta", "beta", "loss", "child_loss", "ridge_effective", "n_right", "n_iters", "stop_reason",
          "failure", "flags", "fallback_iteration", "final_alpha", "trace_loss", "trace_step")


def level(seed, K, d=3, R=2):
    rng = np.random.default_rng(seed)
    ns = rng.integers(0, 700, K)
    ns[0] = 900
    Xs = [rng.uniform(-1, 1, (n, d)) for n in ns]
    ys = [np.tanh(4 * (X @ rng.normal(size=d))) + 0.1 * X[:, 0] for X in Xs]
    th0 = rng.normal(size=(K, R, d + 1))
    th0[..., d] = 0.0
    ro = np.concatenate([[0], np.cumsum(ns)])
    return ns, np.concatenate([X.reshape(-1) for X in Xs]), np.concatenate(ys), ro, th0


def test_graph_replay_equals_eager_across_levels():
    from art import AffineRidgeModel
    from art.graphs import SplitLevelGraphs
    from art.splitters import SoftObliqueSplitter, split_level

    sp = SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 0.1, max_iters=15, n_restarts=2, min_side_points=3,
                             min_side_fraction=0.0)
    graphs = SplitLevelGraphs()
    classes = set()
    for seed, K in ((1, 5), (2, 7), (3, 3), (4, 20)):   # capacities: powers of two >= 8 nodes, >= 4096 rows
        ns, x, y, ro, th0 = level(seed, K)
        kw = dict(parent_loss=np.full(K, 0.5), min_side_fallback=np.zeros(K, np.int8), theta0=th0, traces=True)
        classes.add((max(8, 1 << (K - 1).bit_length()), max(4096, 1 << (int(ro[-1]) - 1).bit_length())))
        eager = split_level(sp, x, y, ro, [3] * K, [O.AFFINE] * K, 0.1, 1e-6, max_dim=3, max_features=4, **kw)
        eager = {f: getattr(eager, f).cpu().numpy() for f in FIELDS}
        got = graphs.split_level(sp, x, y, ro, [3] * K, [O.AFFINE] * K, 0.1, 1e-6, max_dim=3, max_features=4, **kw)
        for f in FIELDS:
            np.testing.assert_array_equal(getattr(got, f).cpu().numpy(), eager[f], err_msg=f"{seed} {f}")
    assert graphs.captures == len(classes) < 4 and graphs.replays == 4


def test_bfs_build_with_graphs_equals_build_without():
    from art import (AffineRidgeModel, BoxDomain, HitAndRunSampler, RegressionTreeBuilder, SoftObliqueSplitter,
                     SplitNode, TemperatureConfig)

    def f(X):
        X = np.atleast_2d(X)
        return np.sin(3 * X[:, 0]) + np.tanh(6 * (X[:, 1] - 0.2 * X[:, 0]))

    def build(graphs):
        model = AffineRidgeModel(ridge=1e-6)
        sp = SoftObliqueSplitter(model, 0.05, max_iters=30, min_side_points=8, min_side_fraction=0.0)
        return RegressionTreeBuilder(domain=BoxDomain.hypercube(2, -1.0, 1.0), oracle=f, model_template=model,
                                     splitter=sp, error_threshold=0.02, max_depth=4, sample_count=300,
                                     temperature_config=TemperatureConfig(strategy="splitter"), random_state=5,
                                     oracle_vectorized=True, traversal="bfs", cuda_graphs=graphs,
                                     isotropic_sampling=False,
                                     sampler=HitAndRunSampler(burn_in=0, thinning=3, rng_mode="device")).build()

    a, b = build(True), build(False)
    na, nb = list(a.tree.iter_nodes()), list(b.tree.iter_nodes())
    assert [n.node_id for n in na] == [n.node_id for n in nb] and len(na) > 5
    for u, v in zip(na, nb):
        if isinstance(u, SplitNode):
            np.testing.assert_array_equal(np.r_[u.w, u.z], np.r_[v.w, v.z])
        else:
            np.testing.assert_array_equal(u.model.coef_, v.model.coef_)


@pytest.mark.parametrize("isotropic", [False, True])
def test_cohort_top_up_equals_one_child_at_a_time(isotropic):
    """BFS children topped up in one hit-and-run launch per cohort (two with
    covariance-shaped sampling: pilots, then main chains with per-child
    direction maps) get the samples, and hence the tree, of the one-at-a-time
    top-up."""

    from art import (AffineRidgeModel, BoxDomain, HitAndRunSampler, RegressionTreeBuilder, SoftObliqueSplitter,
                     SplitNode, TemperatureConfig)

    def f(X):
        X = np.atleast_2d(X)
        return np.exp(-4 * ((X[:, 0] - 0.3) ** 2 + X[:, 1] ** 2)) + 0.5 * np.tanh(5 * X[:, 1])

    def build(cohort):
        model = AffineRidgeModel(ridge=1e-6)
        sp = SoftObliqueSplitter(model, 0.05, max_iters=25, min_side_points=8, min_side_fraction=0.0)
        b = RegressionTreeBuilder(domain=BoxDomain.hypercube(2, -1.0, 1.0), oracle=f, model_template=model,
                                  splitter=sp, error_threshold=0.01, max_depth=4, sample_count=400,
                                  temperature_config=TemperatureConfig(strategy="splitter"), random_state=9,
                                  oracle_vectorized=True, traversal="bfs", cohort_top_up=cohort,
                                  isotropic_sampling=isotropic,
                                  sampler=HitAndRunSampler(burn_in=0, thinning=4, rng_mode="device"))
        return b.build()

    a, b = build(True), build(False)
    assert a.oracle_queries == b.oracle_queries
    na, nb = list(a.tree.iter_nodes()), list(b.tree.iter_nodes())
    assert [n.node_id for n in na] == [n.node_id for n in nb] and len(na) > 5
    for u, v in zip(na, nb):
        if isinstance(u, SplitNode):
            np.testing.assert_array_equal(np.r_[u.w, u.z], np.r_[v.w, v.z])
        else:
            np.testing.assert_array_equal(u.model.coef_, v.model.coef_)
