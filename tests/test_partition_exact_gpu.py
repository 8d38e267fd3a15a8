"""Side decisions at the split plane: (x.w - z) >= 0 goes right
(builder.py:494, tree.py:159, splitters.py:618).

The device decides by the sign of the exact value of x.w - z (a compensated
dot product, and exact expansion arithmetic where its error bound cannot
decide).  Points are placed within ~1e-15 of the plane, and exactly on it,
so the rounded score numpy computes often has the wrong sign.  Each check
compares the device with exact rational arithmetic (fractions.Fraction):
the partition (art_partition_rows), the split kernel's hard partition count,
and tree routing (art_tree_predict) must equal it for every point.  Every
disagreement with numpy's (X @ w - z) >= 0 must then be a point where
numpy's rounded score has the wrong sign -- never a real disagreement."""

from fractions import Fraction

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def exact_right(X, w, z):
    W = [Fraction(float(v)) for v in w]
    Z = Fraction(float(z))
    return np.array([sum(Fraction(float(a)) * b for a, b in zip(row, W)) - Z >= 0 for row in X])


def near_plane_points(rng, w, z, n, d):
    base = rng.uniform(-1, 1, (n, d))
    X = base - ((base @ w) - z)[:, None] * w[None, :]          # on the plane up to rounding
    k = rng.integers(-8, 9, n)
    X = X + (k * 1e-16)[:, None] * w[None, :]                   # spread within ~1e-15
    far = rng.uniform(-1, 1, (n // 4, d))                        # and some ordinary points
    X = np.vstack([X, far])
    # a few points exactly on the plane: x = t * e_0 with w_0 x_0 = z exactly
    if w[0] != 0.0:
        on = np.zeros((4, d))
        on[:, 0] = z / w[0]
        ok = np.array([Fraction(float(v)) * Fraction(float(w[0])) == Fraction(float(z)) for v in on[:, 0]])
        X = np.vstack([X, on[ok]])
    return X


@pytest.mark.parametrize("d", [2, 5, 16, 64])
def test_partition_and_routing_equal_exact_arithmetic_near_the_plane(d):
    from art.tree import partition_rows

    rng = np.random.default_rng(100 + d)
    w = rng.normal(size=d)
    w /= np.linalg.norm(w)
    z = float(rng.uniform(-0.3, 0.3))
    X = near_plane_points(rng, w, z, 3000, d)
    n = X.shape[0]
    ex = exact_right(X, w, z)
    theta = np.r_[w, z][None, :]
    perm, n_right = partition_rows(X.reshape(-1), [0, n], [d], theta)
    perm, nr = perm.cpu().numpy(), int(n_right.cpu().numpy()[0])
    assert nr == int(ex.sum())
    right_rows = np.sort(perm[n - nr:])
    np.testing.assert_array_equal(right_rows, np.flatnonzero(ex))
    assert np.all(np.diff(perm[: n - nr]) > 0) and np.all(np.diff(perm[n - nr:]) > 0)   # stable
    # numpy's rounded score: every disagreement is numpy's own rounding
    npy = (X @ w - z) >= 0.0
    dis = np.flatnonzero(npy != ex)
    assert d <= 2 or dis.size > 0          # the set does exercise rounding-flipped points
    for i in dis:
        assert npy[i] != ex[i]             # numpy wrong, exact arithmetic (= device) right


@pytest.mark.parametrize("d", [3, 16])
def test_split_kernel_hard_partition_counts_exact_sides(d):
    """max_iters = 0: the hard partition of the (projected) start plane; its
    right-side count equals the exact count for the plane the kernel reports."""
    from art import AffineRidgeModel, SoftObliqueSplitter
    from art.splitters import split_level

    rng = np.random.default_rng(7 + d)
    w = rng.normal(size=d)
    w /= np.linalg.norm(w)
    z = float(rng.uniform(-0.2, 0.2))
    X = near_plane_points(rng, w, z, 2000, d)
    n = X.shape[0]
    y = rng.normal(size=n)
    s = SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 0.1, max_iters=0, min_side_points=1,
                            min_side_fraction=0.0)
    res = split_level(s, X.reshape(-1), y, [0, n], [d], [0], 0.1, 1e-6, parent_loss=[1.0],
                      theta0=np.r_[w, z][None, None, :], hard_refit=False)
    th = res.theta.cpu().numpy()[0]
    ex = exact_right(X, th[:d], th[d])
    assert int(res.n_right.cpu().numpy()[0]) == int(ex.sum())


def test_tree_routing_equals_exact_sides():
    from art import AffineRidgeModel
    from art.tree import LeafNode, RegressionTree, SplitNode

    d = 4
    rng = np.random.default_rng(77)
    w = rng.normal(size=d)
    w /= np.linalg.norm(w)
    z = 0.1
    X = near_plane_points(rng, w, z, 2000, d)
    left, right = AffineRidgeModel(), AffineRidgeModel()
    left.coef_ = np.r_[np.zeros(d), -1.0]
    right.coef_ = np.r_[np.zeros(d), 1.0]
    box = None
    root = SplitNode(node_id="0", depth=0, region=box, w=w, z=z,
                     left=LeafNode(node_id="0L", depth=1, region=box, model=left),
                     right=LeafNode(node_id="0R", depth=1, region=box, model=right))
    tree = RegressionTree(root)
    leaf, pred = tree.predict_device(X)
    ex = exact_right(X, w, z)
    np.testing.assert_array_equal(pred, np.where(ex, 1.0, -1.0))
