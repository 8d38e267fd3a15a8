"""Batched weighted ridge on the GPU vs the oracle and the reference's golden outputs.

Tolerance (FP64 plain form): relative coefficient error
    ||beta - beta_ref|| / ||beta_ref|| <= max(1e-10, 1e-14 * cond)
where cond is the 2-norm condition number of G + lambda I: two FP64 solvers
with different summation orders agree to about cond * 1e-16, so a fixed 1e-10
holds for every system with cond <= 1e4 and the bound grows with cond above.
"""

import numpy as np
import pytest

from conftest import GOLDEN, gpu_available
from oracle import ridge as O

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cond_of(phi, w, lam_rel, floor=1e-12):
    sw = np.maximum(w, floor)
    G = phi.T @ (phi * sw[:, None])
    lam = lam_rel * np.trace(G) / G.shape[0]
    return float(np.linalg.cond(G + lam * np.eye(G.shape[0])))


def tol_for(cond):
    return max(1e-10, 1e-14 * cond)


def golden_cases():
    g = np.load(GOLDEN / "ridge_golden.npz")
    for i in range(int(g["count"])):
        kind, lam, solver = g[f"c{i}_meta"]
        yield dict(X=g[f"c{i}_X"], y=g[f"c{i}_y"], w=g[f"c{i}_w"], kind=int(kind), ridge=float(lam),
                   solver=("normal", "auto", "qr", "svd")[int(solver)], beta=g[f"c{i}_beta"],
                   ridge_eff=float(g[f"c{i}_ridge_eff"]), solver_used=str(g[f"c{i}_solver_used"]),
                   cond=float(g[f"c{i}_cond"]), rank=int(g[f"c{i}_rank"]))


@pytest.mark.parametrize("case", list(golden_cases()), ids=lambda c: f"{c['solver']}-k{c['kind']}-n{len(c['y'])}")
def test_single_solves_match_reference_golden(case):
    """Every reference solver (normal, auto with its QR fallback, qr, svd):
    coefficients at max(1e-10, 1e-14 cond); for svd also the rank and the
    2-norm condition number of the augmented design (1e-9 relative: the
    singular values of R against LAPACK's of the whole design).  A rank-
    deficient svd case (ridge 0, a column equal to the sum of two others)
    compares gelsd's minimum-norm solution at 1e-9."""
    from art import models

    res = models._solve_single(case["X"], case["y"], case["w"], case["ridge"], case["kind"],
                               weight_floor=1e-12, solver=case["solver"], auto_rcond_threshold=1e-10)
    phi = O.features(case["X"], case["kind"])
    if case["solver_used"] == "svd" and case["rank"] < phi.shape[1]:
        tol = 1e-9
    else:
        tol = tol_for(cond_of(phi, case["w"], case["ridge"]))
    assert rel_err(res.coefficients, case["beta"]) <= tol
    assert res.ridge_effective == pytest.approx(case["ridge_eff"], rel=1e-12, abs=1e-300)
    assert res.solver_used == case["solver_used"]
    if case["solver_used"] == "svd":
        assert res.rank == case["rank"]
        assert res.condition_estimator == "svd_2norm"
        if np.isfinite(case["cond"]) and case["rank"] == phi.shape[1]:
            assert res.cond_estimate == pytest.approx(case["cond"], rel=1e-9)


def test_batched_svd_solver_matches_gelsd_on_mixed_segments():
    """solver="svd" over a batch of every feature class (9 to 153 features):
    the Jacobi SVD of R against the oracle's gelsd, at max(1e-10, 1e-14 cond)."""
    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    wl = make_batch(K=48, seed=23, n_max=400)
    out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                       x_offsets=wl.x_offsets, solver="svd", precision="fp64",
                                       max_features=wl.max_features, max_dim=wl.max_dim, condition=True)
    beta, status = out.beta.cpu().numpy(), out.status.cpu().numpy()
    info, cond = out.info.cpu().numpy(), out.cond_estimate.cpu().numpy()
    assert set(wl.kinds.tolist()) and max(int(p) for p in wl.dims) == 16
    for k in range(wl.count):
        r0, r1 = wl.row_offsets[k], wl.row_offsets[k + 1]
        d = int(wl.dims[k])
        X = wl.x[wl.x_offsets[k]: wl.x_offsets[k] + (r1 - r0) * d].reshape(-1, d)
        phi = O.features(X, int(wl.kinds[k]))
        p = phi.shape[1]
        ref = O.solve_weighted_ridge(phi, wl.y[r0:r1], wl.w[r0:r1], wl.ridge[k], solver="svd")
        assert status[k] == 0 and info[k] & N.INFO_SVD
        assert (int(info[k]) >> N.INFO_RANK_SHIFT) & 0xFF == ref["rank"]
        c = cond_of(phi, wl.w[r0:r1], wl.ridge[k])
        assert rel_err(beta[k, :p], ref["coefficients"]) <= tol_for(c), (k, p, c)
        assert cond[k] == pytest.approx(ref["cond_estimate"], rel=1e-8)


def test_auto_falls_back_to_svd_when_the_qr_solution_is_not_finite():
    """A zero feature column and no ridge: the Cholesky fails, the unpivoted
    QR meets a zero pivot, and the auto solver re-solves by the SVD
    (models.py:426-438).  The zero column's coefficient is 0 and the others
    equal the reference's least-squares solution."""
    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    rng = np.random.default_rng(31)
    X = np.column_stack([rng.uniform(-1, 1, 50), np.zeros(50), rng.uniform(-1, 1, 50)])
    y = X[:, 0] - 2 * X[:, 2] + 0.01 * rng.normal(size=50)
    out = solve_weighted_ridge_batched(X.reshape(-1), y, None, [0, 50], [3], [N.FEATURES_POLY1_NOBIAS], [0.0],
                                       solver="auto", precision="fp64", max_features=3, max_dim=3, condition=True)
    info = int(out.info.cpu().numpy()[0])
    assert out.status.cpu().numpy()[0] == 0
    assert info & N.INFO_SVD and info & N.INFO_QR_FALLBACK
    assert (info >> N.INFO_RANK_SHIFT) & 0xFF == 2
    ref = O.solve_weighted_ridge(X, y, np.ones(50), 0.0, solver="svd")["coefficients"]
    np.testing.assert_allclose(out.beta.cpu().numpy()[0], ref, rtol=1e-10, atol=1e-12)
    assert out.beta.cpu().numpy()[0, 1] == 0.0


def make_batch(K=96, seed=7, n_max=700):
    from art import workloads

    return workloads.ridge_systems(K, seed=seed, n_min=1, n_max=n_max)


@pytest.mark.parametrize("solver", ["normal", "auto"])
def test_batched_fp64_matches_oracle_on_mixed_segments(solver):
    from art.models import solve_weighted_ridge_batched

    wl = make_batch()
    out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                       x_offsets=wl.x_offsets, solver=solver, precision="fp64",
                                       max_features=wl.max_features, max_dim=wl.max_dim)
    beta = out.beta.cpu().numpy()
    status = out.status.cpu().numpy()
    lam = out.ridge_effective.cpu().numpy()
    for k in range(wl.count):
        r0, r1 = wl.row_offsets[k], wl.row_offsets[k + 1]
        d = int(wl.dims[k])
        X = wl.x[wl.x_offsets[k]: wl.x_offsets[k] + (r1 - r0) * d].reshape(-1, d)
        phi = O.features(X, int(wl.kinds[k]))
        p = phi.shape[1]
        try:
            ref = O.solve_weighted_ridge(phi, wl.y[r0:r1], wl.w[r0:r1], wl.ridge[k], solver=solver)
        except np.linalg.LinAlgError:
            assert status[k] > 0
            continue
        assert status[k] == 0, (k, status[k])
        assert lam[k] == pytest.approx(ref["ridge_effective"], rel=1e-12)
        c = cond_of(phi, wl.w[r0:r1], wl.ridge[k])
        assert rel_err(beta[k, :p], ref["coefficients"]) <= tol_for(c), (k, c)


def test_batched_is_deterministic_and_ordering_independent():
    import torch

    from art.models import solve_weighted_ridge_batched

    wl = make_batch(K=40, seed=11)
    a = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                     x_offsets=wl.x_offsets, max_features=wl.max_features, max_dim=wl.max_dim)
    b = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                     x_offsets=wl.x_offsets, max_features=wl.max_features, max_dim=wl.max_dim)
    assert torch.equal(torch.nan_to_num(a.beta, nan=7.0), torch.nan_to_num(b.beta, nan=7.0))
    # a system solved alone equals the same system inside the batch, bit for bit
    from art.models import kind_feature_count

    for k in (0, 5, 17):
        sub = wl.subset([k])
        c = solve_weighted_ridge_batched(sub.x, sub.y, sub.w, sub.row_offsets, sub.dims, sub.kinds, sub.ridge,
                                         x_offsets=sub.x_offsets, max_features=wl.max_features, max_dim=wl.max_dim)
        p = kind_feature_count(int(wl.dims[k]), int(wl.kinds[k]))
        np.testing.assert_array_equal(c.beta.cpu().numpy()[0, :p], a.beta.cpu().numpy()[k, :p])
        assert np.isnan(c.beta.cpu().numpy()[0, p:]).all()


def test_edge_cases_status_codes():
    from art.models import solve_weighted_ridge_batched

    rng = np.random.default_rng(5)
    # systems: empty, one row, NaN x, negative weight, singular (ridge 0), unsupported d
    d = 3
    n = [0, 1, 10, 10, 10, 10]
    X = rng.uniform(-1, 1, (sum(n), d))
    X[1 + 2] = np.nan  # first row of system 2
    y = rng.normal(size=sum(n))
    w = np.ones(sum(n))
    w[1 + 10 + 4] = -1.0  # system 3
    X[21:31, 1] = 0.0    # system 4: zero column, ridge 0 -> singular
    ro = np.concatenate([[0], np.cumsum(n)])
    dims = np.array([d, d, d, d, d, 99])
    kinds = np.zeros(6, dtype=np.int32)
    ridge = np.array([1e-3, 1e-3, 1e-3, 1e-3, 0.0, 1e-3])
    xo = ro[:-1] * d
    out = solve_weighted_ridge_batched(X.reshape(-1), y, w, ro, dims, kinds, ridge, x_offsets=xo,
                                       max_features=4, max_dim=d)
    st = out.status.cpu().numpy()
    assert st[0] == 1          # empty: G = 0, lambda = 0 -> first pivot fails
    assert st[1] in (0, 2)     # one row, rank 1 + ridge: pivot 2 may still be tiny but positive
    assert st[2] == -2         # non-finite x
    assert st[3] == -1         # negative weight
    assert st[4] == 2          # zero second column, no ridge
    assert st[5] == -4         # d outside the compiled limit
    beta = out.beta.cpu().numpy()
    assert np.isnan(beta[2]).all() and np.isnan(beta[4]).all()


def test_auto_solver_qr_fallback_reports_info_bits():
    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    rng = np.random.default_rng(16)
    base = rng.normal(size=120)
    X = np.column_stack([base, base + 1e-7 * rng.normal(size=120), rng.normal(size=120)])
    y = rng.normal(size=120)
    out = solve_weighted_ridge_batched(X.reshape(-1), y, None, [0, 120], [3], [N.FEATURES_POLY1_NOBIAS],
                                       [0.0], solver="auto", max_features=3, max_dim=3)
    info = int(out.info.cpu().numpy()[0])
    assert info & N.INFO_QR_FALLBACK
    ref = O.solve_weighted_ridge(X, y, np.ones(120), 0.0, solver="auto")
    assert ref["solver_used"] == "qr"
    c = np.linalg.cond(X.T @ X)
    assert rel_err(out.beta.cpu().numpy()[0], ref["coefficients"]) <= max(1e-10, 1e-14 * c)


def test_models_fit_on_gpu_match_oracle():
    from art import AffineRidgeModel, PolynomialRidgeModel

    rng = np.random.default_rng(21)
    X = rng.uniform(-1, 1, (300, 4))
    y = np.cos(X[:, 0]) + X[:, 1] * X[:, 2]
    w = rng.uniform(0.1, 1, 300)
    m = AffineRidgeModel(ridge=1e-6).fit_weighted(X, y, w)
    ref = O.solve_weighted_ridge(O.features(X, O.AFFINE), y, w, 1e-6)
    assert rel_err(m.coef_, ref["coefficients"]) < 1e-11
    pm = PolynomialRidgeModel(degree=2, ridge=1e-8).fit(X, y)
    ref = O.solve_weighted_ridge(O.features(X, O.POLY2), y, np.ones(300), 1e-8)
    assert rel_err(pm.coef_, ref["coefficients"]) < 1e-9
    np.testing.assert_allclose(pm.predict(X), O.features(X, O.POLY2) @ ref["coefficients"], rtol=1e-8, atol=1e-9)


# ----------------------------------------------------------- mixed precision
def _oracle_check(wl, out, solver="normal"):
    beta = out.beta.cpu().numpy()
    status = out.status.cpu().numpy()
    worst = 0.0
    for k in range(wl.count):
        r0, r1 = wl.row_offsets[k], wl.row_offsets[k + 1]
        d = int(wl.dims[k])
        X = wl.x[wl.x_offsets[k]: wl.x_offsets[k] + (r1 - r0) * d].reshape(-1, d)
        phi = O.features(X, int(wl.kinds[k]))
        p = phi.shape[1]
        try:
            ref = O.solve_weighted_ridge(phi, wl.y[r0:r1], wl.w[r0:r1], wl.ridge[k], solver=solver)
        except np.linalg.LinAlgError:
            assert status[k] > 0
            continue
        assert status[k] == 0, (k, status[k])
        c = cond_of(phi, wl.w[r0:r1], wl.ridge[k])
        err = rel_err(beta[k, :p], ref["coefficients"])
        assert err <= tol_for(c), (k, p, c, err)
        worst = max(worst, err / tol_for(c))
    return worst


@pytest.mark.parametrize("seed,K,n_max", [(7, 96, 700), (8, 24, 5000)])
def test_batched_mixed_matches_oracle(seed, K, n_max):
    """Mixed form (tcgen05 TF32x3 Gram, FP32 Cholesky, FP64 refinement) meets the
    same FP64 tolerance as the plain form; systems it cannot refine are re-solved."""

    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    wl = make_batch(K=K, seed=seed, n_max=n_max)
    out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                       x_offsets=wl.x_offsets, precision="mixed",
                                       max_features=wl.max_features, max_dim=wl.max_dim)
    _oracle_check(wl, out)
    info = out.info.cpu().numpy()
    p = np.array([O.feature_count(int(d), int(k)) for d, k in zip(wl.dims, wl.kinds)])
    tensor = p >= 33
    resolved = np.mean((info[tensor] & N.INFO_FP64_RESOLVE) != 0)
    passes = (info[tensor] >> N.INFO_REFINE_SHIFT) & 255
    print(f"mixed: resolved {resolved:.3f}, mean refinement passes {passes.mean():.2f}")


@pytest.mark.parametrize("seed,K,n_max", [(7, 96, 700), (8, 24, 5000)])
def test_batched_mixed_fp64_factor_matches_oracle(seed, K, n_max):
    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    wl = make_batch(K=K, seed=seed, n_max=n_max)
    out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                       x_offsets=wl.x_offsets, precision="mixed", fp64_factor=True,
                                       max_features=wl.max_features, max_dim=wl.max_dim)
    _oracle_check(wl, out)
    info = out.info.cpu().numpy()
    p = np.array([O.feature_count(int(d), int(k)) for d, k in zip(wl.dims, wl.kinds)])
    tensor = p >= 33
    resolved = np.mean((info[tensor] & N.INFO_FP64_RESOLVE) != 0)
    print(f"mixed/fp64 factor: resolved {resolved:.3f}")


def test_tensor_core_gram_accuracy():
    """TF32 hi/lo split products, FP32 accumulation in chains of at most 256 rows
    summed in FP32: ||G' - G||_F <= 3e-6 ||G||_F for every system."""

    from art.models import ridge_gram_batched

    wl = make_batch(K=32, seed=13, n_max=3000)
    gram, status = ridge_gram_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds,
                                      x_offsets=wl.x_offsets, max_features=wl.max_features, max_dim=wl.max_dim)
    gram = gram.cpu().numpy().astype(float)
    status = status.cpu().numpy()
    checked = 0
    errs = []
    for k in range(wl.count):
        r0, r1 = wl.row_offsets[k], wl.row_offsets[k + 1]
        d = int(wl.dims[k])
        p = O.feature_count(d, int(wl.kinds[k]))
        if p < 33:
            assert status[k] == -4
            continue
        assert status[k] == 0
        X = wl.x[wl.x_offsets[k]: wl.x_offsets[k] + (r1 - r0) * d].reshape(-1, d)
        phi = O.features(X, int(wl.kinds[k]))
        q = np.maximum(wl.w[r0:r1], 1e-12)
        G = phi.T @ (phi * q[:, None])
        il = np.tril_indices(p)
        Gd = np.zeros((p, p))
        packed = gram[k, : p * (p + 1) // 2]
        rows, cols = [], []
        for i in range(p):
            rows += [i] * (i + 1)
            cols += list(range(i + 1))
        Gd[rows, cols] = packed
        Gd = Gd + np.tril(Gd, -1).T
        err = np.linalg.norm(Gd - G) / np.linalg.norm(G)
        print(f"system {k} p={p} n={r1 - r0} rel Frobenius error {err:.2e}")
        errs.append((k, p, err))
        checked += 1
    assert checked >= 5
    worst = max(errs, key=lambda e: e[2])
    assert worst[2] <= 3e-6, worst


def test_mixed_is_deterministic_and_alone_equals_batched():
    from art.models import kind_feature_count, solve_weighted_ridge_batched

    wl = make_batch(K=40, seed=12)
    kw = dict(x_offsets=wl.x_offsets, precision="mixed", max_features=wl.max_features, max_dim=wl.max_dim)
    a = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge, **kw)
    b = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge, **kw)
    np.testing.assert_array_equal(np.nan_to_num(a.beta.cpu().numpy()), np.nan_to_num(b.beta.cpu().numpy()))
    for k in range(wl.count):
        if O.feature_count(int(wl.dims[k]), int(wl.kinds[k])) >= 33:
            break
    sub = wl.subset([k])
    kw["x_offsets"] = sub.x_offsets
    c = solve_weighted_ridge_batched(sub.x, sub.y, sub.w, sub.row_offsets, sub.dims, sub.kinds, sub.ridge, **kw)
    p = kind_feature_count(int(wl.dims[k]), int(wl.kinds[k]))
    np.testing.assert_array_equal(c.beta.cpu().numpy()[0, :p], a.beta.cpu().numpy()[k, :p])


def test_mixed_edge_cases_fall_back_to_fp64_statuses():
    from art.models import solve_weighted_ridge_batched

    rng = np.random.default_rng(9)
    d, n = 8, [0, 50, 50]
    X = rng.uniform(-1, 1, (sum(n), d))
    X[3, 2] = np.inf
    y = rng.normal(size=sum(n))
    w = np.ones(sum(n))
    w[60] = -2.0
    ro = np.concatenate([[0], np.cumsum(n)])
    out = solve_weighted_ridge_batched(X.reshape(-1), y, w, ro, [d] * 3, [2] * 3, [1e-4] * 3,
                                       precision="mixed", max_features=45, max_dim=d)
    st = out.status.cpu().numpy()
    assert st[0] == 1 and st[1] == -2 and st[2] == -1


def test_tensor_threshold_routes_feature_classes():
    """The mixed form's tensor-core threshold only moves systems between kernels:
    every routing meets the oracle tolerance, and systems below the threshold
    carry no refinement passes (FP64 kernels)."""

    from art import _native as N
    from art.models import solve_weighted_ridge_batched

    wl = make_batch(K=64, seed=11, n_max=900)
    p = np.array([O.feature_count(int(d), int(k)) for d, k in zip(wl.dims, wl.kinds)])
    for threshold in (33, 46, 161):
        out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                           x_offsets=wl.x_offsets, precision="mixed",
                                           max_features=wl.max_features, max_dim=wl.max_dim,
                                           tensor_min_features=threshold)
        _oracle_check(wl, out)
        passes = (out.info.cpu().numpy() >> N.INFO_REFINE_SHIFT) & 255
        assert np.all(passes[p < threshold] == 0), threshold


def test_autotuned_threshold_is_stored_and_used():
    from art import autotune
    from art.models import solve_weighted_ridge_batched

    autotune.clear()
    try:
        wl = make_batch(K=64, seed=12, n_max=1500)
        entry = autotune.tune_ridge_threshold(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                              x_offsets=wl.x_offsets, max_dim=wl.max_dim, per_class=16,
                                              repeats=1)
        assert entry["tensor_min_features"] in (45, 153, autotune.NO_TENSOR)
        assert set(entry["classes"]) == {"45", "153"}
        assert autotune.cached_ridge_threshold() == entry["tensor_min_features"]
        out = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, wl.row_offsets, wl.dims, wl.kinds, wl.ridge,
                                           x_offsets=wl.x_offsets, precision="mixed",
                                           max_features=wl.max_features, max_dim=wl.max_dim)
        _oracle_check(wl, out)
    finally:
        autotune.clear()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_host_inputs_staged_in_slices_equal_one_copy(precision):
    """Host (pinned) inputs cut into slices whose copies overlap the solves
    give exactly the coefficients and statuses of one copy followed by one
    solve, and of device-resident inputs."""
    import torch

    from art import _native as N
    from art import workloads
    from art.models import solve_weighted_ridge_batched

    wl = workloads.ridge_systems(600, seed=9, n_min=32, n_max=900)
    hx, hy, hw = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (wl.x, wl.y, wl.w))
    args = (wl.row_offsets, wl.dims, wl.kinds, wl.ridge)
    kw = dict(x_offsets=wl.x_offsets, precision=precision, max_features=wl.max_features, max_dim=wl.max_dim,
              tensor_min_features=45)
    one = solve_weighted_ridge_batched(hx, hy, hw, *args, host_slices=1, **kw)
    staged = solve_weighted_ridge_batched(hx, hy, hw, *args, host_slices=7, **kw)
    dev = solve_weighted_ridge_batched(hx.cuda(), hy.cuda(), hw.cuda(), *args, **kw)
    for res in (staged, dev):
        np.testing.assert_array_equal(res.status.cpu().numpy(), one.status.cpu().numpy())
        np.testing.assert_array_equal(res.beta.cpu().numpy(), one.beta.cpu().numpy())
        np.testing.assert_array_equal(res.ridge_effective.cpu().numpy(), one.ridge_effective.cpu().numpy())
    assert (one.status.cpu().numpy() == 0).mean() > 0.95
    # numpy inputs take the same staged path (synchronous copies)
    np_staged = solve_weighted_ridge_batched(wl.x, wl.y, wl.w, *args, host_slices=3, **kw)
    np.testing.assert_array_equal(np_staged.beta.cpu().numpy(), one.beta.cpu().numpy())
