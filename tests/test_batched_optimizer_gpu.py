"""BatchedOptimizerWorkspace / optimize_batch (the reference's resident
batched optimizer API, _cuda_batched_optimizer.py:88-660) over the device
split search.  Given starts, every node's split equals the oracle's
restatement of SoftObliqueSplitter.split at the FP64 form's tolerances
(split parameters 1e-9 relative, identical stop reasons, iteration counts
and partitions); slot selection, return order and validation follow the
reference."""

import numpy as np
import pytest

from conftest import gpu_available
from oracle import ridge as O
from oracle import split as S

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _cohort(K=5, n=180, d=3, seed=3):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (K, n, d))
    y = np.empty((K, n))
    for k in range(K):
        a = rng.normal(size=d)
        a /= np.linalg.norm(a)
        y[k] = np.tanh(5 * (X[k] @ a - 0.1)) + 0.2 * X[k, :, 0] ** 2 + 0.01 * rng.normal(size=n)
    th0 = np.array([S.initialize_theta(X[k], rng) for k in range(K)])
    return X, y, th0


def _splitter(R=1, **kw):
    from art import AffineRidgeModel, SoftObliqueSplitter

    return SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 0.1, max_iters=20, n_restarts=R, min_side_points=10,
                               min_side_fraction=0.0, **kw)


def _oracle(X, y, th, T=0.1, R=1):
    p = S.Params(max_iters=20, n_restarts=R, min_side_points=10, min_side_fraction=0.0)
    phi = O.features(X, O.AFFINE)
    beta = O.solve_weighted_ridge(phi, y, np.ones(len(y)), 1e-6)["coefficients"]
    parent = float(np.mean((y - phi @ beta) ** 2))
    return S.split(X, y, th if np.ndim(th) == 2 else [th], T, O.AFFINE, 1e-6, parent, p), parent


def test_workspace_equals_oracle_split_per_node_in_slot_order():
    from art import BatchedOptimizerWorkspace, SplitResult

    X, y, th0 = _cohort()
    temps = np.array([0.1, 0.1, 0.1, 0.1, 0.1])
    ws = BatchedOptimizerWorkspace.allocate(_splitter(), capacity=8, n=X.shape[1], d=X.shape[2])
    ws.load(X, y, temperature=temps)
    order = [3, 0, 4]
    out = ws.optimize(th0[order], nodes=order)
    assert len(out) == 3
    for res, j in zip(out, order):
        assert isinstance(res, SplitResult)
        ref, parent = _oracle(X[j], y[j], th0[j])
        np.testing.assert_allclose(np.r_[res.w, res.z], np.r_[ref["w"], ref["z"]], rtol=1e-9, atol=1e-11)
        assert res.stop_reason == ref["stop_reason"] and res.n_iters == ref["n_iters"]
        assert res.n_right == ref["n_right"]
        assert res.parent_loss == pytest.approx(parent, rel=1e-10)
        np.testing.assert_allclose(res.loss, ref["loss"], rtol=1e-9)
    ws.close()
    with pytest.raises(RuntimeError):
        ws.optimize(th0)


def test_optimize_batch_with_parent_losses_and_device_starts():
    from art import SplitNotFoundError, SplitResult, optimize_batch

    X, y, th0 = _cohort(seed=8)
    a = optimize_batch(_splitter(), X, y, theta0=th0, parent_loss=np.ones(5))
    for k, res in enumerate(a):
        ref, _ = _oracle(X[k], y[k], th0[k])
        np.testing.assert_allclose(np.r_[res.w, res.z], np.r_[ref["w"], ref["z"]], rtol=1e-9, atol=1e-11)
        assert res.parent_loss == 1.0
    # device-drawn starts, two restarts: valid unit-normal splits with both sides populated
    b = optimize_batch(_splitter(R=2), X, y)
    for res in b:
        assert isinstance(res, (SplitResult, SplitNotFoundError))
        if isinstance(res, SplitResult):
            assert np.linalg.norm(res.w) == pytest.approx(1.0, rel=1e-12)
            assert res.n_left + res.n_right == X.shape[1] and min(res.n_left, res.n_right) >= 10


def test_two_dimensional_start_with_restarts_and_validation():
    from art import BatchedOptimizerWorkspace

    X, y, th0 = _cohort(seed=9)
    with BatchedOptimizerWorkspace(_splitter(R=3), X, y) as ws:
        out = ws.optimize(th0)       # restart 0 from th0, restarts 1, 2 drawn
        assert len(out) == 5
        with pytest.raises(ValueError):
            ws.optimize(th0, nodes=[0, 0])
        with pytest.raises(ValueError):
            ws.optimize(th0, nodes=[7])
        with pytest.raises(ValueError):
            ws.optimize(th0, hard_refit=False)      # needs n_restarts == 1
        with pytest.raises(ValueError):
            ws.optimize(np.zeros((5, 2)))
        with pytest.raises(ValueError):
            ws.load(X[:, :, :2], y)
    with pytest.raises(ValueError):
        BatchedOptimizerWorkspace(_splitter(), X, y, temperature=-1.0)
