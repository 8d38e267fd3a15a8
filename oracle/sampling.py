"""Oracle: hit-and-run transitions (reference art/_numba_sampling.py,
art/sampling.py) -- test infrastructure only.

``chains_batched`` restates sample_precomputed_chains(_parallel)
(_numba_sampling.py:45-167): unnormalised directions, slack updated
incrementally, exact-zero product tests, a sample after every `thinning`
steps following `burn_in`.  ``chain_scalar`` restates HitAndRunSampler.sample
(sampling.py:445-495) with its _step_interval (540-564).  Both take injected
draws.  ``autocorrelation_by_lag`` restates sampling.py:214-256.
"""

from __future__ import annotations

import numpy as np


def chains_batched(A, b, x0, directions, uniforms, burn_in, thinning, n_rounds):
    """A (m,d), b (m,), x0 (C,d), directions (C,steps,d), uniforms (C,steps).

    Returns samples (n_rounds, C, d) and final points (C, d).
    """
    x = np.array(x0, dtype=float, copy=True)
    slack = b[None, :] - x @ A.T                       # sampling.py:648
    Au = directions @ A.T                              # sampling.py:875-884
    C = x.shape[0]
    out = np.empty((n_rounds, C, x.shape[1]))
    step = 0

    def advance(step):
        prod = Au[:, step, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = slack / prod
        t_lo = np.max(np.where(prod < 0.0, ratio, -np.inf), axis=1)
        t_hi = np.min(np.where(prod > 0.0, ratio, np.inf), axis=1)
        t = t_lo + uniforms[:, step] * (t_hi - t_lo)
        x[:] += t[:, None] * directions[:, step, :]
        slack[:] -= t[:, None] * prod

    for _ in range(burn_in):
        advance(step)
        step += 1
    for r in range(n_rounds):
        for _ in range(thinning):
            advance(step)
            step += 1
        out[r] = x
    return out, x


def chain_scalar(A, b, x0, directions, uniforms, burn_in, thinning, n, tol=1e-10):
    """HitAndRunSampler.sample with injected draws (one chain)."""
    x = np.asarray(x0, float).copy()
    samples = []
    ucur = 0
    for step in range(burn_in + n * thinning):
        d = directions[step]
        nrm = np.linalg.norm(d)
        if nrm == 0.0:
            continue
        d = d / nrm
        Ax = A @ x
        Ad = A @ d
        slack = b - Ax
        pos = Ad > 1e-14
        neg = Ad < -1e-14
        if np.any(~(pos | neg) & (slack < -tol)):
            raise RuntimeError("Current point is infeasible.")
        ratios = np.zeros_like(Ad)
        np.divide(slack, Ad, out=ratios, where=pos | neg)
        t_lo = np.max(ratios, where=neg, initial=-np.inf)
        t_hi = np.min(ratios, where=pos, initial=np.inf)
        if t_lo > t_hi:
            raise RuntimeError("Empty hit-and-run step interval.")
        t = t_lo + uniforms[ucur] * (t_hi - t_lo)
        ucur += 1
        x = x + t * d
        if step >= burn_in and (step - burn_in) % thinning == 0:
            samples.append(x.copy())
    return np.asarray(samples)


def box_rows(lo, hi):
    """BoxDomain.as_region rows (domain.py:87-92): [I; -I] x <= [hi; -lo]."""
    d = len(lo)
    return np.vstack([np.eye(d), -np.eye(d)]), np.concatenate([hi, -np.asarray(lo)])


def autocorrelation_by_lag(series, lags):
    """sampling.py:214-256"""
    values = np.asarray(series, float)
    if values.ndim == 1:
        values = values[:, None]
    centered = values - values.mean(axis=0, keepdims=True)
    scales = np.max(np.abs(centered), axis=0)
    nonconst = scales > 0
    norm = np.zeros_like(centered)
    np.divide(centered, scales, out=norm, where=nonconst)
    var = np.mean(norm * norm, axis=0)
    out = np.zeros((len(lags), values.shape[1]))
    for i, lag in enumerate(lags):
        cov = np.mean(norm[:-lag] * norm[lag:], axis=0)
        out[i] = np.divide(cov, var, out=np.zeros_like(cov), where=nonconst)
    return out


def rejection_sample(A, b, lo, hi, n, rng):
    """Exactly uniform points of {lo <= x <= hi, A x <= b} by rejection."""
    d = len(lo)
    out = []
    while sum(len(o) for o in out) < n:
        X = rng.uniform(lo, hi, size=(max(4 * n, 1024), d))
        keep = np.all(X @ A.T <= b[None, :], axis=1) if len(b) else np.ones(len(X), bool)
        out.append(X[keep])
    return np.concatenate(out)[:n]
