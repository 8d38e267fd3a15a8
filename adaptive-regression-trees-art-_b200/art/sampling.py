"""Hit-and-run sampling in node polytopes on the GPU.

Drop-in for the reference ``art/sampling.py``: ``HitAndRunSampler``
(sampling.py:432-564), ``BatchedHitAndRunSampler`` and its numba variants
(601-1025) and the host helpers.  Chains run in ``art_hit_and_run``; box rows
(``+-e_i``) are applied structurally, every other row densely, all in FP64.

Random draws come from one of two sources:

* ``rng_mode="reference"`` -- the directions and chord uniforms are drawn on
  the host from ``random_state`` in exactly the order the reference consumes
  its generator, then injected; the chain then equals the reference chain
  to rounding (the parity mode used by the tree builder's parity tests).
* ``rng_mode="device"`` -- counter-based Philox4x32-10 on the device, keyed
  per chain from ``random_state`` (the fast mode).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace
from typing import ClassVar, Literal, Protocol, Sequence, runtime_checkable

import numpy as np

from . import _native as N
from ._device import ptr, require_cuda, stream_handle, to_device, torch
from .domain import BoxDomain, PolytopeRegion

RandomState = int | np.random.Generator | None
RngMode = Literal["reference", "device"]


def as_rng(random_state: RandomState = None) -> np.random.Generator:
    if isinstance(random_state, np.random.Generator):
        return random_state
    return np.random.default_rng(random_state)


@runtime_checkable
class Sampler(Protocol):
    def sample(self, region: PolytopeRegion, n: int, random_state: RandomState = None,
               x0: np.ndarray | None = None) -> np.ndarray: ...


def sample_uniform_box(bounds: np.ndarray, n: int, random_state: RandomState = None) -> np.ndarray:
    """sampling.py:67-83 (host; the root of a box domain)."""

    bounds = np.asarray(bounds, dtype=float)
    if bounds.ndim != 2 or bounds.shape[1] != 2:
        raise ValueError(f"bounds must have shape (d, 2), got {bounds.shape}.")
    if np.any(bounds[:, 0] >= bounds[:, 1]):
        raise ValueError("Each bound must satisfy low < high.")
    if n < 0:
        raise ValueError("n must be nonnegative.")
    return as_rng(random_state).uniform(bounds[:, 0], bounds[:, 1], size=(int(n), bounds.shape[0]))


def sample_covariance_eigendecomposition(samples, *, assume_centered: bool = False):
    """sampling.py:86-106."""

    values = np.asarray(samples, dtype=float)
    if values.ndim != 2:
        raise ValueError(f"samples must have shape (n_samples, d), got {values.shape}.")
    if values.shape[0] < 2:
        raise ValueError("samples must contain at least two points.")
    if not np.all(np.isfinite(values)):
        raise ValueError("samples must contain only finite values.")
    centered = values if assume_centered else values - values.mean(axis=0, keepdims=True)
    cov = centered.T @ centered / (centered.shape[0] - 1)
    eigenvalues, eigenvectors = np.linalg.eigh(cov)
    return eigenvectors, eigenvalues


def covariance_eigendecomposition_batched(sample_sets, *, stream=None):
    """``sample_covariance_eigendecomposition`` for many point sets of one
    dimension in one device launch (``art_covariance_eigh``): returns a list
    of (eigenvectors, eigenvalues) host arrays, eigenvalues ascending and
    eigenvector j in column j as numpy's ``eigh``.  Each eigenvector's
    largest-magnitude component is positive (numpy's signs are LAPACK's),
    and values agree with ``eigh`` to rounding.  Raises like the host form
    for sets of fewer than two points or with non-finite values."""

    t = torch()
    dev = require_cuda()
    sets = [np.asarray(v, dtype=float) for v in sample_sets]
    if not sets:
        return []
    d = sets[0].shape[1] if sets[0].ndim == 2 else -1
    for v in sets:
        if v.ndim != 2 or v.shape[1] != d:
            raise ValueError("every sample set must have shape (n_samples, d) with one d.")
        if v.shape[0] < 2:
            raise ValueError("samples must contain at least two points.")
        if not np.all(np.isfinite(v)):
            raise ValueError("samples must contain only finite values.")
    lib = N.load_library()
    x = to_device(np.concatenate(sets).reshape(-1), t.float64, dev)
    ro = to_device(np.concatenate([[0], np.cumsum([v.shape[0] for v in sets])]).astype(np.int64), t.int64, dev)
    K = len(sets)
    vals = t.empty((K, d), dtype=t.float64, device=dev)
    vecs = t.empty((K, d, d), dtype=t.float64, device=dev)
    status = t.empty(K, dtype=t.int32, device=dev)
    N.check(lib.art_covariance_eigh(ptr(x), ptr(ro), K, d, ptr(vals), ptr(vecs), ptr(status), stream_handle(stream)),
            "art_covariance_eigh")
    st = status.cpu().numpy()
    if np.any(st != 0):
        raise RuntimeError(f"covariance eigendecomposition failed for set(s) {np.flatnonzero(st != 0).tolist()} "
                           f"(status {st[st != 0].tolist()}).")
    vals_h, vecs_h = vals.cpu().numpy(), vecs.cpu().numpy()
    return [(vecs_h[k], vals_h[k]) for k in range(K)]


def floor_covariance_eigenvalues(eigenvalues, floor_ratio: float):
    """sampling.py:109-127."""

    values = np.asarray(eigenvalues, dtype=float).reshape(-1)
    if values.size == 0:
        raise ValueError("eigenvalues must contain at least one value.")
    if not np.all(np.isfinite(values)):
        raise ValueError("eigenvalues must be finite.")
    if not np.isfinite(floor_ratio) or floor_ratio <= 0.0:
        raise ValueError("floor_ratio must be positive.")
    mean = float(np.mean(values))
    if mean <= 0.0:
        raise ValueError("eigenvalues must have a positive mean before flooring.")
    floor = float(floor_ratio * mean)
    return np.maximum(values, floor), floor


def infer_box_bounds(region: PolytopeRegion, tol: float = 1e-12):
    """sampling.py:145-167."""

    lows = np.full(region.dimension, -np.inf)
    highs = np.full(region.dimension, np.inf)
    for row, bound in zip(region.A, region.b):
        nz = np.flatnonzero(np.abs(row) > tol)
        if nz.size != 1:
            continue
        i = int(nz[0])
        coef = row[i]
        if coef > 0:
            highs[i] = min(highs[i], bound / coef)
        else:
            lows[i] = max(lows[i], bound / coef)
    if np.any(~np.isfinite(lows)) or np.any(~np.isfinite(highs)) or np.any(lows >= highs):
        return None
    return np.column_stack([lows, highs])


def find_feasible_point(region: PolytopeRegion, bounds=None, max_tries: int = 20000,
                        random_state: RandomState = None, tol: float = 1e-10) -> np.ndarray:
    """sampling.py:170-190 (host rejection sampling for a chain start)."""

    if bounds is None:
        bounds = infer_box_bounds(region)
    if bounds is None:
        raise ValueError("bounds are required when they cannot be inferred from the region.")
    rng = as_rng(random_state)
    for _ in range(max_tries):
        x = sample_uniform_box(bounds, 1, random_state=rng)[0]
        if bool(region.contains(x, tol=tol)[0]):
            return x
    raise RuntimeError("Could not find a feasible point inside the region.")


def autocorrelation_by_lag(series: np.ndarray, lags: Sequence[int]) -> np.ndarray:
    """Signed autocorrelation per lag and series (sampling.py:214-256; host diagnostic)."""

    values = np.asarray(series, dtype=float)
    if values.ndim == 1:
        values = values.reshape(-1, 1)
    if values.ndim != 2:
        raise ValueError("series must have shape (n_steps,) or (n_steps, n_series).")
    if values.shape[0] < 2:
        raise ValueError("series must contain at least two states.")
    if not np.all(np.isfinite(values)):
        raise ValueError("series must contain only finite values.")
    lags_array = np.asarray(lags, dtype=int).reshape(-1)
    if lags_array.size == 0:
        raise ValueError("lags must contain at least one value.")
    if np.any(lags_array < 1) or np.any(lags_array >= values.shape[0]):
        raise ValueError("lags must lie in [1, n_steps).")
    centered = values - np.mean(values, axis=0, keepdims=True)
    scales = np.max(np.abs(centered), axis=0)
    nonconstant = scales > 0.0
    normalized = np.zeros_like(centered)
    np.divide(centered, scales, out=normalized, where=nonconstant)
    variance = np.mean(normalized * normalized, axis=0)
    out = np.zeros((lags_array.size, values.shape[1]))
    for i, lag in enumerate(lags_array):
        cov = np.mean(normalized[:-lag] * normalized[lag:], axis=0)
        out[i] = np.divide(cov, variance, out=np.zeros_like(cov), where=nonconstant)
    return out


# ------------------------------------------------------------------ device
@dataclass
class DevicePolytopes:
    """Polytopes in the kernel layout: box bounds + oblique CSR rows (torch CUDA)."""

    dim: int
    lo: object
    hi: object
    row_offsets: object
    A: object
    b: object
    max_rows: int
    maps: object = None   # [count][d][d] direction maps (covariance-shaped sampling) or None

    @property
    def count(self) -> int:
        return int(self.lo.shape[0])


def split_box_rows(A: np.ndarray, b: np.ndarray):
    """Separate exact +-e_i rows (box bounds) from the other (oblique) rows.

    A row equal to +e_i bounds x_i <= b, a row equal to -e_i bounds
    x_i >= -b; for those rows A u = +-u_i exactly, so structural handling is
    bit-identical to the dense product.  Later duplicates stay oblique.
    """

    A = np.asarray(A, float)
    b = np.asarray(b, float)
    d = A.shape[1]
    lo = np.full(d, -np.inf)
    hi = np.full(d, np.inf)
    has_lo = np.zeros(d, bool)
    has_hi = np.zeros(d, bool)
    keep = np.ones(A.shape[0], bool)
    for r in range(A.shape[0]):
        nz = np.flatnonzero(A[r])
        if nz.size != 1:
            continue
        i = int(nz[0])
        if A[r, i] == 1.0 and not has_hi[i]:
            hi[i], has_hi[i], keep[r] = b[r], True, False
        elif A[r, i] == -1.0 and not has_lo[i]:
            lo[i], has_lo[i], keep[r] = -b[r], True, False
    return lo, hi, A[keep], b[keep]


def device_polytopes(regions: Sequence[PolytopeRegion] | Sequence[tuple], maps=None) -> DevicePolytopes:
    """Pack regions (or (A, b) pairs) for ``art_hit_and_run``; ``maps`` gives
    one d x d direction map per region (device draws become u = M z)."""

    t = torch()
    dev = require_cuda()
    los, his, As, bs, offs = [], [], [], [], [0]
    d = None
    for reg in regions:
        A, b = (reg.A, reg.b) if isinstance(reg, PolytopeRegion) else reg
        lo, hi, Ao, bo = split_box_rows(A, b)
        d = A.shape[1] if d is None else d
        if A.shape[1] != d:
            raise ValueError("all polytopes of one call must share the dimension")
        los.append(lo)
        his.append(hi)
        As.append(Ao)
        bs.append(bo)
        offs.append(offs[-1] + Ao.shape[0])
    max_rows = max((a.shape[0] for a in As), default=0)
    if max_rows > 32:
        raise ValueError("at most 32 non-box rows per polytope are supported")
    Acat = np.concatenate(As) if offs[-1] else np.zeros((1, d))
    bcat = np.concatenate(bs) if offs[-1] else np.zeros(1)
    return DevicePolytopes(
        d, to_device(np.stack(los), t.float64, dev), to_device(np.stack(his), t.float64, dev),
        to_device(np.asarray(offs, np.int64), t.int64, dev), to_device(Acat, t.float64, dev),
        to_device(bcat, t.float64, dev), max_rows,
        None if maps is None else to_device(np.ascontiguousarray(np.stack(maps), dtype=float), t.float64, dev))


def hit_and_run_device(polys: DevicePolytopes, chain_polytope, x0, *, burn_in: int, thinning: int,
                       n_rounds: int, mode: str = "batched", seeds=None, directions=None,
                       uniforms=None, counter_base: int = 0, stream=None):
    """Advance chains on the device.  Returns (samples[n_rounds, C, d], last x[C, d], status[C])."""

    t = torch()
    lib = N.load_library()
    dev = require_cuda()
    x = to_device(x0, t.float64, dev).clone()
    Cn = int(x.shape[0])
    cp = to_device(chain_polytope, t.int32, dev)
    samples = t.empty((max(n_rounds, 0), Cn, polys.dim), dtype=t.float64, device=dev)
    status = t.empty(Cn, dtype=t.int32, device=dev)
    sd = None if seeds is None else to_device(np.asarray(seeds, dtype=np.uint64).view(np.int64) if not isinstance(seeds, t.Tensor) else seeds, t.int64, dev)
    dr = None if directions is None else to_device(directions, t.float64, dev)
    un = None if uniforms is None else to_device(uniforms, t.float64, dev)
    P = N.ArtPolytopes(polys.count, polys.dim, ptr(polys.lo), ptr(polys.hi), ptr(polys.row_offsets),
                       ptr(polys.A), ptr(polys.b), polys.max_rows, 0, ptr(polys.maps))
    Ch = N.ArtChains(Cn, ptr(cp), ptr(x), ptr(sd), ptr(dr), ptr(un),
                     N.HAR_SCALAR if mode == "scalar" else N.HAR_BATCHED, int(burn_in), int(thinning),
                     int(n_rounds), int(counter_base), ptr(samples), ptr(status))
    N.check(lib.art_hit_and_run(C.byref(P), C.byref(Ch), stream_handle(stream)), "art_hit_and_run")
    samples._keepalive = (cp, sd, dr, un)
    return samples, x, status


_STATUS_TEXT = {1: "Empty hit-and-run step interval.", 2: "x0 is not feasible for the region.",
                3: "too many polytope rows for the compiled kernel"}


def _raise_status(status):
    st = np.asarray(status)
    bad = st[st != 0]
    if bad.size:
        code = int(bad[0])
        exc = ValueError if code == 2 else RuntimeError
        raise exc(_STATUS_TEXT.get(code, f"hit-and-run status {code}"))


@dataclass
class HitAndRunSampler:
    """Hit-and-run sampler for convex polytopes A x <= b (sampling.py:432-564)."""

    burn_in: int = 500
    thinning: int = 10
    feasibility_tol: float = 1e-10
    max_feasible_tries: int = 20000
    bounds: np.ndarray | None = None
    direction_eigenvectors: np.ndarray | None = None
    direction_eigenvalues: np.ndarray | None = None
    direction_eigenvalue_floor: float = 1e-4
    rng_mode: RngMode = "reference"

    def sample(self, region: PolytopeRegion, n: int, random_state: RandomState = None,
               x0: np.ndarray | None = None) -> np.ndarray:
        if n < 0:
            raise ValueError("n must be nonnegative.")
        if self.burn_in < 0:
            raise ValueError("burn_in must be nonnegative.")
        if self.thinning < 1:
            raise ValueError("thinning must be at least 1.")
        rng = as_rng(random_state)
        vecs, sqrt_vals = self._direction_spectrum(region.dimension)
        if x0 is None:
            x = find_feasible_point(region, bounds=self.bounds, max_tries=self.max_feasible_tries,
                                    random_state=rng, tol=self.feasibility_tol)
        else:
            x = np.asarray(x0, dtype=float).reshape(-1)
            if x.shape[0] != region.dimension:
                raise ValueError(f"x0 must have shape ({region.dimension},), got {x.shape}.")
            if not bool(region.contains(x, tol=self.feasibility_tol)[0]):
                raise ValueError("x0 is not feasible for the region.")
        n = int(n)
        d = region.dimension
        total = self.burn_in + n * self.thinning
        if n == 0:
            return np.empty((0, d))
        polys = device_polytopes([region])
        if self.rng_mode == "reference":
            # the reference interleaves normal(size=d) and uniform() per step
            dirs = np.empty((total, d))
            unif = np.zeros(total)
            u_i = 0
            for step in range(total):
                z = rng.normal(size=d)
                if vecs is not None:
                    z = vecs @ (sqrt_vals * z)
                dirs[step] = z
                if np.linalg.norm(z) != 0.0:
                    unif[u_i] = rng.uniform(0.0, 1.0)
                    u_i += 1
            samples, _, status = hit_and_run_device(
                polys, [0], x[None, :], burn_in=self.burn_in, thinning=self.thinning, n_rounds=n,
                mode="scalar", directions=dirs[None], uniforms=unif[None])
        else:
            if vecs is not None:  # covariance-shaped directions: u = vecs diag(sqrt_vals) z on the device
                polys = device_polytopes([region], maps=[vecs * sqrt_vals[None, :]])
            seed = int(rng.integers(0, 2**63 - 1))
            samples, _, status = hit_and_run_device(
                polys, [0], x[None, :], burn_in=self.burn_in, thinning=self.thinning, n_rounds=n,
                mode="scalar", seeds=[seed])
        _raise_status(status.cpu().numpy())
        return samples[:, 0, :].cpu().numpy()

    def sample_many(self, regions, ns, random_states, x0s, spectra=None) -> list:
        """``sample`` for several regions of one dimension in one launch.

        Device draws only (``rng_mode="device"``; the sampler itself has no
        direction spectrum, item k may bring one in ``spectra[k]`` as an
        (eigenvectors, eigenvalues) pair).  Item k is what the matching
        single ``sample`` call returns, or the exception it raises: each chain
        is keyed by the seed its own random state yields, and a chain's first
        n samples do not depend on how many more it runs.  A chain that
        reports a failure is rerun alone, which reproduces the single call.
        """

        if self.rng_mode != "device" or self.direction_eigenvectors is not None \
                or self.direction_eigenvalues is not None:
            raise ValueError("sample_many needs rng_mode='device' and isotropic directions")
        if self.burn_in < 0:
            raise ValueError("burn_in must be nonnegative.")
        if self.thinning < 1:
            raise ValueError("thinning must be at least 1.")
        out: list = [None] * len(regions)
        live = []
        singles = {}
        for k, (reg, n, rs, x0) in enumerate(zip(regions, ns, random_states, x0s)):
            n = int(n)
            if n < 0:
                out[k] = ValueError("n must be nonnegative.")
                continue
            single = self
            mp = None
            if spectra is not None and spectra[k] is not None:
                single = replace(self, direction_eigenvectors=spectra[k][0], direction_eigenvalues=spectra[k][1])
                try:
                    vecs, sv = single._direction_spectrum(reg.dimension)
                except ValueError as exc:
                    out[k] = exc
                    continue
                mp = vecs * sv[None, :]
            singles[k] = single
            rng = as_rng(rs)
            x = np.asarray(x0, dtype=float).reshape(-1)
            if x.shape[0] != reg.dimension:
                out[k] = ValueError(f"x0 must have shape ({reg.dimension},), got {x.shape}.")
                continue
            if not bool(reg.contains(x, tol=self.feasibility_tol)[0]):
                out[k] = ValueError("x0 is not feasible for the region.")
                continue
            if n == 0:
                out[k] = np.empty((0, reg.dimension))
                continue
            live.append((k, reg, n, x, int(rng.integers(0, 2**63 - 1)), mp))
        if not live:
            return out
        maps = None
        if any(it[5] is not None for it in live):
            d = live[0][1].dimension
            maps = [np.eye(d) if it[5] is None else it[5] for it in live]
        polys = device_polytopes([it[1] for it in live], maps=maps)
        samples, _, status = hit_and_run_device(
            polys, np.arange(len(live)), np.stack([it[3] for it in live]), burn_in=self.burn_in,
            thinning=self.thinning, n_rounds=max(it[2] for it in live), mode="scalar",
            seeds=[it[4] for it in live])
        st = status.cpu().numpy()
        host = samples.cpu().numpy()
        for c, (k, reg, n, x, _, _) in enumerate(live):
            if st[c] != 0:
                try:
                    out[k] = singles[k].sample(reg, n, random_state=random_states[k], x0=x0s[k])
                except (RuntimeError, ValueError) as exc:
                    out[k] = exc
            else:
                out[k] = host[:n, c, :].copy()
        return out

    def _direction_spectrum(self, dimension: int):
        vecs, vals = self.direction_eigenvectors, self.direction_eigenvalues
        if vecs is None and vals is None:
            return None, None
        if vecs is None or vals is None:
            raise ValueError("direction_eigenvectors and direction_eigenvalues must be provided together.")
        vecs = np.asarray(vecs, dtype=float)
        vals = np.asarray(vals, dtype=float).reshape(-1)
        if vecs.shape != (dimension, dimension) or vals.shape != (dimension,):
            raise ValueError("direction spectrum shape mismatch")
        if not np.allclose(vecs.T @ vecs, np.eye(dimension), rtol=1e-8, atol=1e-10):
            raise ValueError("direction_eigenvectors must be orthonormal.")
        safe, _ = floor_covariance_eigenvalues(vals, self.direction_eigenvalue_floor)
        s = np.sqrt(safe)
        return vecs, s / np.max(s)


@dataclass
class BatchedHitAndRunSampler(HitAndRunSampler):
    """Several chains with incremental slacks (sampling.py:601-962), on the GPU.

    Chains advance together; ``n`` samples are taken round-robin over the
    chains exactly as the reference lays them out (round-major).
    """

    n_chains: int = 20
    rng_mode: RngMode = "device"
    # layout of the reference's draws: step-major (BatchedHitAndRunSampler,
    # NumbaBatchedHitAndRunSampler) or chain-major (the parallel numba form)
    _chain_major: ClassVar[bool] = False

    def sample(self, region: PolytopeRegion, n: int, random_state: RandomState = None,
               x0: np.ndarray | None = None) -> np.ndarray:
        """sampling.py:643-813.  ``rng_mode="reference"`` draws every
        direction and chord uniform from ``random_state`` exactly as the
        reference class does (the same generator calls, in the same order
        and layout, including the tail round for ``n`` not a multiple of the
        chain count) and injects them, so the samples equal the reference's
        to rounding; ``"device"`` keys counter-based device draws per chain."""

        if n < 0:
            raise ValueError("n must be nonnegative.")
        if self.burn_in < 0:
            raise ValueError("burn_in must be nonnegative.")
        if self.thinning < 0:
            raise ValueError("thinning must be nonnegative.")
        if self.n_chains < 1:
            raise ValueError("n_chains must be at least 1.")
        n = int(n)
        d = region.dimension
        if n == 0:
            return np.empty((0, d))
        rng = as_rng(random_state)
        n_chains = min(self.n_chains, n)
        points = self._initial_points(region, n_chains, rng, x0)
        stride = max(1, self.thinning)
        full_rounds, remainder = divmod(n, n_chains)
        polys = device_polytopes([region])
        if self.rng_mode == "reference":
            return self._sample_reference_draws(polys, points, rng, d, stride, full_rounds, remainder, n)
        vecs, sqrt_vals = self._direction_spectrum(d)
        if vecs is not None:  # covariance-shaped directions: u = vecs diag(sqrt_vals) z on the device
            polys = device_polytopes([region], maps=[vecs * sqrt_vals[None, :]])
        seeds = rng.integers(0, 2**63 - 1, size=n_chains, dtype=np.int64).astype(np.uint64)
        rounds = full_rounds + (1 if remainder else 0)
        samples, _, status = hit_and_run_device(
            polys, np.zeros(n_chains, np.int32), points, burn_in=self.burn_in, thinning=stride,
            n_rounds=rounds, mode="batched", seeds=seeds)
        _raise_status(status.cpu().numpy())
        return samples.reshape(-1, d)[:n].cpu().numpy()

    def _sample_reference_draws(self, polys, points, rng, d, stride, full_rounds, remainder, n):
        n_chains = points.shape[0]
        steps = self.burn_in + full_rounds * stride
        dirs, unif = self._reference_draws(rng, n_chains, steps, d)
        tail = self._reference_draws(rng, remainder, stride, d) if remainder else None
        samples, last, status = hit_and_run_device(
            polys, np.zeros(n_chains, np.int32), points, burn_in=self.burn_in, thinning=stride,
            n_rounds=full_rounds, mode="batched", directions=dirs, uniforms=unif)
        _raise_status(status.cpu().numpy())
        out = [samples.reshape(-1, d)]
        if tail is not None:
            # the first `remainder` chains take one more thinned round (burn-in 0)
            extra, _, status = hit_and_run_device(
                polys, np.zeros(remainder, np.int32), last[:remainder], burn_in=0, thinning=stride,
                n_rounds=1, mode="batched", directions=tail[0], uniforms=tail[1])
            _raise_status(status.cpu().numpy())
            out.append(extra.reshape(-1, d))
        return torch().cat(out)[:n].cpu().numpy()

    def _reference_draws(self, rng, n_chains: int, steps: int, d: int):
        """Directions (chains, steps, d) and uniforms (chains, steps), chain-major,
        from the generator calls of _draw_random_arrays (sampling.py:864-873,
        983-1025) and _shape_directions."""

        if self._chain_major and getattr(self, "parallel_random", False):
            if self.random_threads < 1:
                raise ValueError("random_threads must be at least 1.")
            workers = min(self.random_threads, n_chains)
            dirs = np.empty((n_chains, steps, d))
            unif = np.empty((n_chains, steps))
            seeds = rng.integers(0, np.iinfo(np.uint64).max, size=workers, dtype=np.uint64)
            block, extra = divmod(n_chains, workers)
            start = 0
            for w, seed in enumerate(seeds):
                stop = start + block + (w < extra)
                g = np.random.Generator(np.random.SFC64(int(seed)))
                g.standard_normal(out=dirs[start:stop])
                g.random(out=unif[start:stop])
                start = stop
        elif self._chain_major:
            dirs = rng.normal(size=(n_chains, steps, d))
            unif = rng.random(size=(n_chains, steps))
        else:
            dirs = rng.normal(size=(steps, n_chains, d)).transpose(1, 0, 2)
            unif = rng.random(size=(steps, n_chains)).T
        vecs, sqrt_vals = self._direction_spectrum(d)
        if vecs is not None:
            dirs = (dirs * sqrt_vals) @ vecs.T
        return np.ascontiguousarray(dirs), np.ascontiguousarray(unif)

    def _initial_points(self, region, n_chains, rng, x0):
        """sampling.py:826-862."""

        if x0 is None:
            seed = find_feasible_point(region, bounds=self.bounds, max_tries=self.max_feasible_tries,
                                       random_state=rng, tol=self.feasibility_tol)
            return np.repeat(seed[None, :], n_chains, axis=0)
        cands = np.asarray(x0, dtype=float)
        if cands.ndim == 1:
            cands = cands[None, :]
        if cands.ndim != 2 or cands.shape[1] != region.dimension:
            raise ValueError("x0 must have shape (d,) or (n_points, d)")
        if cands.shape[0] == 0:
            raise ValueError("x0 must contain at least one starting point.")
        if not np.all(region.contains(cands, tol=self.feasibility_tol)):
            raise ValueError("All x0 candidates must be feasible for the region.")
        idx = rng.choice(cands.shape[0], size=n_chains, replace=cands.shape[0] < n_chains)
        return cands[idx].copy()


@dataclass
class NumbaBatchedHitAndRunSampler(BatchedHitAndRunSampler):
    """Name kept from the reference (sampling.py:965-970); runs the same GPU chains."""


@dataclass
class ParallelNumbaBatchedHitAndRunSampler(NumbaBatchedHitAndRunSampler):
    """Name kept from the reference (sampling.py:973-1025); runs the same GPU chains."""

    n_chains: int = 50
    parallel_random: bool = True
    random_threads: int = 10
    _chain_major: ClassVar[bool] = True


@dataclass
class UniformBoxSampler:
    """Exact uniform sampler for axis-aligned boxes (sampling.py:130-142)."""

    def sample(self, domain: BoxDomain, n: int, random_state: RandomState = None, x0=None) -> np.ndarray:
        del x0
        return sample_uniform_box(domain.bounds, n, random_state=random_state)
