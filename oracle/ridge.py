"""Oracle: weighted trace-scaled ridge (reference art/models.py:200-448) -- test infrastructure only.

Restates solve_weighted_ridge with the same scipy/LAPACK calls the reference
makes (cho_factor, dpocon, cho_solve, lstsq with gelsy/gelsd), plus the
feature bases of AffineRidgeModel (bias last, models.py:200-206) and
PolynomialRidgeModel (sklearn order, models.py:571-620).
"""

from __future__ import annotations

from itertools import combinations_with_replacement

import numpy as np

AFFINE, POLY1, POLY2, POLY1_NOBIAS, POLY2_NOBIAS = 0, 1, 2, 3, 4


def features(X: np.ndarray, kind: int) -> np.ndarray:
    """Feature matrix for the kernel feature kinds (art/_cuda_features.py:13-29 order)."""

    X = np.asarray(X, dtype=float)
    n, d = X.shape
    one = np.ones((n, 1))
    if kind == AFFINE:
        return np.hstack([X, one])
    cols = []
    if kind in (POLY1, POLY2):
        cols.append(one)
    cols.append(X)
    if kind in (POLY2, POLY2_NOBIAS):
        cols.append(np.stack([X[:, i] * X[:, j] for i, j in combinations_with_replacement(range(d), 2)], 1)
                    if d else np.zeros((n, 0)))
    return np.hstack(cols)


def feature_count(d: int, kind: int) -> int:
    return {AFFINE: d + 1, POLY1: d + 1, POLY1_NOBIAS: d,
            POLY2: 1 + d + d * (d + 1) // 2, POLY2_NOBIAS: d + d * (d + 1) // 2}[kind]


def solve_weighted_ridge(design, y, weights, ridge, weight_floor=1e-12, solver="normal",
                         auto_rcond_threshold=1e-10):
    """models.py:218-371.  Returns a dict with the RidgeSolveResult fields.

    solver='normal' raises numpy.linalg.LinAlgError on Cholesky failure, as
    the reference does (models.py:283-288).
    """

    from scipy import linalg
    from scipy.linalg import lapack

    design = np.asarray(design, dtype=float)
    y = np.asarray(y, dtype=float).reshape(-1)
    weights = np.asarray(weights, dtype=float).reshape(-1)
    safe = np.maximum(weights, float(weight_floor))                      # :245-247
    if solver in ("qr", "svd"):                                          # :359-371
        ridge_eff = float(ridge) * float(np.sum((design * np.sqrt(safe)[:, None]) ** 2)) / design.shape[1]
        return _augmented(design, y, safe, ridge_eff, solver, solver, None, None, None)
    gram = design.T @ (design * safe[:, None])                           # :253
    rhs = design.T @ (y * safe)                                          # :254
    ridge_eff = float(ridge) * float(np.trace(gram)) / gram.shape[0]      # :271, :209-215
    reg = gram.copy()
    reg.flat[:: gram.shape[0] + 1] += ridge_eff
    gram_norm = linalg.norm(reg, 1, check_finite=False)
    try:
        factor = linalg.cho_factor(reg, lower=True, overwrite_a=True, check_finite=False)
    except linalg.LinAlgError as exc:                                    # :282-306
        if solver == "normal":
            raise np.linalg.LinAlgError("Normal-equation Cholesky factorization failed") from exc
        return _augmented(design, y, safe, ridge_eff, solver, "qr", "cholesky_failure", np.inf,
                          "cholesky_failed")
    rcond, info = lapack.dpocon(factor[0], gram_norm, uplo="L")          # :307-314
    if info == 0 and rcond > 0.0:
        cond = float(np.sqrt(1.0 / min(float(rcond), 1.0)))
        estimator = "sqrt_gram_1norm"
    else:
        rcond, cond, estimator = 0.0, np.inf, "condition_estimate_failure"
    if solver == "normal" or rcond >= auto_rcond_threshold:              # :334-343
        coef = linalg.cho_solve(factor, rhs, check_finite=False)
        return dict(coefficients=coef, solver_requested=solver, solver_used="cholesky",
                    condition_estimator=estimator, cond_estimate=cond, ridge_effective=ridge_eff,
                    rank=None, fallback_reason=None)
    return _augmented(design, y, safe, ridge_eff, solver, "qr", estimator, cond,
                      "rcond_below_threshold")                          # :345-357


def _augmented(design, y, safe, ridge_eff, requested, used, estimator, cond, reason):
    """_solve_augmented_ridge (models.py:374-448)."""

    from scipy import linalg

    sw = np.sqrt(safe)
    A = design * sw[:, None]
    b = y * sw
    if ridge_eff > 0.0:
        A = np.vstack([A, np.sqrt(ridge_eff) * np.eye(design.shape[1])])
        b = np.concatenate([b, np.zeros(design.shape[1])])
    try:
        coef, _, rank, sv = linalg.lstsq(A, b, lapack_driver="gelsy" if used == "qr" else "gelsd",
                                         check_finite=False)
    except linalg.LinAlgError:                                           # :412-424
        if requested != "auto" or used != "qr":
            raise
        return _augmented(design, y, safe, ridge_eff, requested, "svd", None, None, "qr_failed")
    if requested == "auto" and used == "qr" and not np.all(np.isfinite(coef)):  # :426-438
        return _augmented(design, y, safe, ridge_eff, requested, "svd", None, None, "qr_nonfinite")
    if used == "svd":                                                    # :440-442, 455-461
        estimator = "svd_2norm"
        cond = None if sv is None or sv.size == 0 else (np.inf if sv[-1] <= 0.0 else float(sv[0] / sv[-1]))
    return dict(coefficients=coef, solver_requested=requested, solver_used=used,
                condition_estimator=estimator, cond_estimate=cond, ridge_effective=ridge_eff,
                rank=int(rank), fallback_reason=reason)


def solve_segments(x, y, w, row_offsets, dims, kinds, ridge, weight_floor=1e-12, solver="normal",
                   x_offsets=None, max_features=None):
    """Batched convenience loop over node-sorted segments (CSR layout of the kernels).

    Returns (beta[K, max_p] with NaN padding, ridge_eff[K], status[K]) where
    status follows the kernels: 0 ok, >0 Cholesky failure (normal solver).
    """

    K = len(dims)
    p_all = [feature_count(int(d), int(k)) for d, k in zip(dims, kinds)]
    P = max(p_all) if max_features is None else max_features
    beta = np.full((K, P), np.nan)
    lam = np.full(K, np.nan)
    status = np.zeros(K, dtype=np.int32)
    for k in range(K):
        r0, r1 = int(row_offsets[k]), int(row_offsets[k + 1])
        d = int(dims[k])
        xo = r0 * d if x_offsets is None else int(x_offsets[k])
        X = np.asarray(x[xo: xo + (r1 - r0) * d], dtype=float).reshape(r1 - r0, d)
        phi = features(X, int(kinds[k]))
        ww = np.ones(r1 - r0) if w is None else w[r0:r1]
        try:
            res = solve_weighted_ridge(phi, y[r0:r1], ww, float(ridge[k]), weight_floor, solver)
        except np.linalg.LinAlgError:
            status[k] = 1
            continue
        beta[k, : p_all[k]] = res["coefficients"]
        lam[k] = res["ridge_effective"]
    return beta, lam, status
