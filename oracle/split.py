"""Oracle: soft oblique split search (reference art/splitters.py, objectives.py,
optimizers.py) -- test infrastructure only.

A numpy restatement of SoftObliqueSplitter._optimize_from_initialization
(splitters.py:365-601) with the objective of SoftObliqueRidgeObjective
(objectives.py:132-340), armijo_backtracking (optimizers.py:72-121) and
AdaptiveAlpha (optimizers.py:20-69), plus _make_hard_result (603-690),
_initialize_theta (692-700) and restart selection (split, 252-363).  The
optional geometric temperature anneal (T_k = T * ratio^(k/(max_iters-1)),
not in the reference) is applied per accepted iteration when ratio != 1.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import ridge as R


def sigmoid(v):
    """objectives.py:49-51"""
    v = np.clip(v, -50.0, 50.0)
    return 1.0 / (1.0 + np.exp(-v))


def project_unit_w(theta):
    """splitters.py:71-83"""
    theta = np.asarray(theta, dtype=float).reshape(-1)
    n = np.linalg.norm(theta[:-1])
    if n <= 1e-12:
        raise ValueError("Cannot project theta with near-zero w.")
    out = theta.copy()
    out[:-1] = theta[:-1] / n
    return out


def project_unit_w_gradient(theta, grad):
    """splitters.py:86-98"""
    theta = project_unit_w(theta)
    g = np.asarray(grad, dtype=float).copy()
    w = theta[:-1]
    g[:-1] = grad[:-1] - float(grad[:-1] @ w) * w
    return g


@dataclass
class Params:
    max_iters: int = 100
    grad_atol: float = 1e-8
    grad_rtol: float = 1e-5
    min_side_points: int = 1
    min_side_fraction: float = 0.05
    min_side_fallback: bool = False
    n_restarts: int = 1
    alpha0: float = 1.0
    rho: float = 0.5
    armijo_c: float = 1e-4
    max_backtracks: int = 25
    adaptive_alpha: bool = True
    alpha_min: float = 1e-12
    alpha_max: float = 1e3
    alpha_grow: float = 10.0
    alpha_recovery: float = 10.0
    heavy_backtrack_threshold: int = 8
    max_line_search_failures: int = 3
    weight_floor: float = 1e-12
    anneal_ratio: float = 1.0


class AdaptiveAlpha:
    """optimizers.py:20-69"""

    def __init__(self, p: Params):
        self.p = p
        self.alpha = self._clip(p.alpha0)

    def _clip(self, a):
        return min(max(float(a), self.p.alpha_min), self.p.alpha_max)

    def update(self, success, step, nb, rho):
        if not success:
            self.alpha = self._clip(step * rho)
        elif nb == 0:
            self.alpha = self._clip(step * self.p.alpha_grow)
        elif nb >= self.p.heavy_backtrack_threshold:
            self.alpha = self._clip(step * self.p.alpha_recovery)
        else:
            self.alpha = self._clip(step / rho)
        return self.alpha


def armijo(value_fn, candidate_fn, f0, dd, alpha0, rho, c, max_backtracks):
    """optimizers.py:72-121 -> (theta, value, step, success, n_backtracks)"""
    alpha = float(alpha0)
    th = candidate_fn(alpha)
    val = float(value_fn(th))
    for nb in range(max_backtracks + 1):
        if nb > 0:
            alpha *= rho
            th = candidate_fn(alpha)
            val = float(value_fn(th))
        if val <= f0 + c * alpha * dd:
            return th, val, alpha, True, nb
    return th, val, alpha, False, max_backtracks


class Objective:
    """SoftObliqueRidgeObjective (objectives.py:69-360) for a feature kind."""

    def __init__(self, X, y, T, kind, ridge, weight_floor=1e-12):
        self.X = np.asarray(X, float)
        self.y = np.asarray(y, float)
        self.T = float(T)
        self.phi = R.features(self.X, kind)
        self.ridge = ridge
        self.floor = weight_floor

    def fit(self, weights, floor):
        return R.solve_weighted_ridge(self.phi, self.y, weights, self.ridge, weight_floor=floor)["coefficients"]

    def evaluate(self, theta, ref=None):
        w, z = theta[:-1], float(theta[-1])
        pi = sigmoid((self.X @ w - z) / self.T)
        if ref is None:
            bl = self.fit(1.0 - pi, self.floor)
            br = self.fit(pi, self.floor)
            rl = self.y - self.phi @ bl
            rr = self.y - self.phi @ br
        else:
            bl, br, rl, rr = ref["bl"], ref["br"], ref["rl"], ref["rr"]
        loss = float(np.mean((1.0 - pi) * rl ** 2 + pi * rr ** 2))
        return dict(theta=theta.copy(), pi=pi, bl=bl, br=br, rl=rl, rr=rr, loss=loss)

    def grad(self, ev):
        n = self.X.shape[0]
        coeff = (ev["rr"] ** 2 - ev["rl"] ** 2) * ev["pi"] * (1.0 - ev["pi"]) / n
        gw = self.X.T @ coeff / self.T
        gz = -float(np.sum(coeff)) / self.T
        return np.concatenate([gw, [gz]])


def required_side_points(n, p: Params):
    """splitters.py:752-754"""
    return max(int(p.min_side_points), int(np.ceil(p.min_side_fraction * n)))


def initialize_theta(X, rng):
    """splitters.py:692-700"""
    w = rng.normal(size=X.shape[1])
    nrm = np.linalg.norm(w)
    if nrm <= 1e-12:
        w[0] = 1.0
        nrm = 1.0
    w = w / nrm
    return np.concatenate([w, [float(np.median(X @ w))]])


def optimize(X, y, theta0, T, kind, ridge, p: Params):
    """splitters.py:365-601.  Returns a dict with theta, histories, stop reason."""
    obj = Objective(X, y, T, kind, ridge, p.weight_floor)
    n = X.shape[0]
    req = required_side_points(n, p)
    theta = project_unit_w(theta0)
    cur = obj.evaluate(theta)
    g = obj.grad(cur)
    pg = project_unit_w_gradient(theta, g)
    g0 = float(np.linalg.norm(pg))
    tol = p.grad_atol + p.grad_rtol * g0
    nr = int(np.count_nonzero(cur["pi"] >= 0.5))
    last_feasible = theta.copy() if min(nr, n - nr) >= req else None
    last_it = 0 if last_feasible is not None else None
    losses, gnorms, steps, backs = [cur["loss"]], [g0], [], []
    ctl = AdaptiveAlpha(p)
    reason, converged = "max_iters", False
    for it in range(p.max_iters):
        d = -pg
        dd = float(g @ d)
        if gnorms[-1] <= tol:
            converged, reason = True, "gradient_tolerance"
            break
        if dd >= 0.0:
            reason = "non_descent_direction"
            break
        failures = 0
        while True:
            a0 = ctl.alpha if p.adaptive_alpha else p.alpha0
            th, val, step, ok, nb = armijo(lambda t: obj.evaluate(t, ref=cur)["loss"],
                                           lambda a: project_unit_w(theta + a * d), cur["loss"], dd, a0,
                                           p.rho, p.armijo_c, p.max_backtracks)
            if p.adaptive_alpha:
                ctl.update(ok, step, nb, p.rho)
            if ok:
                break
            failures += 1
            if not p.adaptive_alpha:
                reason = "line_search_failed"
                break
            if failures >= p.max_line_search_failures:
                reason = "max_line_search_failures"
                break
            if ctl.alpha <= p.alpha_min:
                reason = "alpha_min_reached"
                break
        if not ok:
            break
        theta = th
        if p.anneal_ratio != 1.0 and p.max_iters > 1:
            obj.T = T * p.anneal_ratio ** ((it + 1) / (p.max_iters - 1))
        cur = obj.evaluate(theta)
        g = obj.grad(cur)
        pg = project_unit_w_gradient(theta, g)
        losses.append(cur["loss"])
        gnorms.append(float(np.linalg.norm(pg)))
        steps.append(step)
        backs.append(nb)
        nr = int(np.count_nonzero(cur["pi"] >= 0.5))
        if min(nr, n - nr) >= req:
            last_feasible, last_it = theta.copy(), len(losses) - 1
    out = dict(theta=theta, losses=losses, grad_norms=gnorms, steps=steps, backtracks=backs,
               stop_reason=reason, converged=converged, n_iters=len(losses) - 1,
               final_alpha=ctl.alpha if p.adaptive_alpha else p.alpha0, fallback=False,
               fallback_iteration=None, tolerance=tol)
    nr = int(np.count_nonzero(cur["pi"] >= 0.5))
    if min(nr, n - nr) < req and p.min_side_fallback and last_feasible is not None:
        out["theta"] = last_feasible
        out["fallback"] = True
        out["fallback_iteration"] = last_it
    return out


def hard_result(X, y, theta, kind, ridge, parent_loss, p: Params, hard_refit=True):
    """splitters.py:603-690 -> dict or raises ValueError('min_side_points')."""
    theta = project_unit_w(theta)
    w, z = theta[:-1], float(theta[-1])
    right = (X @ w - z) >= 0.0
    n = len(y)
    nr = int(right.sum())
    nl = n - nr
    req = required_side_points(n, p)
    if nl < req or nr < req:
        raise ValueError("min_side_points")
    out = dict(w=w.copy(), z=z, n_left=nl, n_right=nr, right=right)
    if not hard_refit:
        return out
    phi = R.features(X, kind)
    bl = R.solve_weighted_ridge(phi[~right], y[~right], np.ones(nl), ridge)["coefficients"]
    br = R.solve_weighted_ridge(phi[right], y[right], np.ones(nr), ridge)["coefficients"]
    ll = float(np.mean((y[~right] - phi[~right] @ bl) ** 2))
    lr = float(np.mean((y[right] - phi[right] @ br) ** 2))
    loss = nl / n * ll + nr / n * lr
    out.update(bl=bl, br=br, left_loss=ll, right_loss=lr, loss=loss, split_gain=parent_loss - loss)
    return out


def split(X, y, theta0s, T, kind, ridge, parent_loss, p: Params, hard_refit=True):
    """Restart loop and selection of SoftObliqueSplitter.split (splitters.py:324-363)."""
    best = best_fb = None
    failure = None
    for th0 in theta0s:
        try:
            opt = optimize(X, y, th0, T, kind, ridge, p)
            hr = hard_result(X, y, opt["theta"], kind, ridge, parent_loss, p, hard_refit)
        except ValueError as exc:
            failure = str(exc)
            continue
        hr.update(opt)
        if not hard_refit:
            return hr  # geometry only (single restart, splitters.py:326-327)
        if opt["fallback"]:
            if best_fb is None or hr["loss"] < best_fb["loss"]:
                best_fb = hr
        elif best is None or hr["loss"] < best["loss"]:
            best = hr
    if best is not None:
        return best
    if best_fb is not None:
        return best_fb
    raise ValueError(failure or "invalid_split")
