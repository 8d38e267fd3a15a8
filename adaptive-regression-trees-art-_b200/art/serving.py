"""Continuous-batching service for surrogate-tree builds on one GPU.

A job is a level-wise regression-tree build over its own seeded samples of a
target function, followed by adaptive rounds that add hit-and-run samples
inside the leaves with the largest fit error.  The service keeps every
job's samples and tree on the device and advances all admitted jobs one
tree level per tick.  Each tick co-batches, across jobs, the work of that
level into single library calls:

  * ``art_ridge_batched``      leaf fits of every frontier node (mixed or FP64),
  * ``art_segment_residuals``  their relative L2 fit errors,
  * ``art_split_level``        the soft oblique split search of the nodes
                               that are neither converged nor at max depth,
  * ``art_partition_rows``     the stable partition of their rows,
  * ``art_hit_and_run``        the refinement samples of a round.

Jobs are admitted as they arrive while both a slot and their HBM footprint
fit the budget, and leave when their last round converges.  Every random
draw is keyed by the job's seed and the node's path (device Philox keys),
and every kernel solves each node independently with a fixed summation
order, so a job's tree is the same whether it runs alone or in a mix.

The node policy is the fixed-sample form of the reference builder
(builder.py:358-551 without per-child top-up): fit, stop on tolerance or
depth, otherwise split and route ``(X @ w - z) >= 0`` to the right.
"""

from __future__ import annotations

import ctypes as C
import hashlib
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .autotune import WARP_MAX_DIM, WARP_MAX_FEATURES

WARP_MAX_ROWS = 1 << 16  # split nodes up to this size take the warp-per-restart form
from ._device import ptr, require_cuda, stream_handle, torch
from .models import AffineRidgeModel, segment_residuals, solve_weighted_ridge_batched
from .splitters import SoftObliqueSplitter, split_level

__all__ = ["SurrogateJob", "JobResult", "ServingEngine", "poisson_jobs", "job_footprint"]


def _key(*parts) -> int:
    """64-bit key of a tuple (stable across runs and processes)."""

    h = hashlib.blake2b(repr(parts).encode(), digest_size=8).digest()
    return int.from_bytes(h, "little")


@dataclass
class SurrogateJob:
    """One surrogate-build request: d-dimensional target, n0 initial samples."""

    job_id: int
    dim: int
    n_initial: int
    seed: int
    arrival: float = 0.0
    max_depth: int = 12
    rounds: int = 3
    grow_fraction: float = 0.1
    refine_leaves: int = 4
    error_threshold: float = 0.02
    min_side_points: int = 0          # 0: twice the feature count
    temperature: float = 0.1
    max_iters: int = 30
    ridge: float = 1e-6

    @property
    def kind(self) -> int:
        """Quadratic leaves for d <= 8, affine otherwise."""
        return N.FEATURES_POLY2 if self.dim <= 8 else N.FEATURES_AFFINE

    @property
    def n_features(self) -> int:
        d = self.dim
        return 1 + d + d * (d + 1) // 2 if self.kind == N.FEATURES_POLY2 else d + 1

    @property
    def n_final(self) -> int:
        per_round = int(round(self.grow_fraction * self.n_initial))
        return self.n_initial + self.rounds * per_round


def job_footprint(job: SurrogateJob) -> int:
    """Device bytes a job holds while admitted: samples, targets and the
    per-tick staging copies (three row-sized buffers)."""

    return int(job.n_final * (job.dim + 1) * 8 * 3 + (1 << 20))


def poisson_jobs(count: int, rate: float, seed: int = 5, dims=(2, 4, 8, 16, 32), n_min: int = 1000,
                 n_max: int = 1_000_000, **kw) -> list[SurrogateJob]:
    """A Poisson stream: exponential inter-arrival times at ``rate`` jobs/s,
    d uniform over ``dims``, n0 log-uniform in [n_min, n_max]."""

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    d = rng.choice(np.asarray(dims), count)
    n = np.floor(np.exp(rng.uniform(np.log(n_min), np.log(n_max), count))).astype(int)
    return [SurrogateJob(job_id=i, dim=int(d[i]), n_initial=int(n[i]), seed=int(rng.integers(1 << 62)),
                         arrival=float(t[i]), **kw) for i in range(count)]


class _Target:
    """f(x) = sum of 8 Gaussian bumps (widths U(0.1, 0.6) sqrt(d/2),
    amplitudes N(0,1)) + tanh(8 (u.x - b)) on the device."""

    def __init__(self, job: SurrogateJob, device):
        t = torch()
        rng = np.random.default_rng([job.seed, 7])
        d = job.dim
        self.c = t.as_tensor(rng.uniform(-1, 1, (8, d)), device=device)
        self.w = t.as_tensor(rng.uniform(0.1, 0.6, 8) * np.sqrt(d / 2.0), device=device)
        self.a = t.as_tensor(rng.normal(size=8), device=device)
        u = rng.normal(size=d)
        self.u = t.as_tensor(u / np.linalg.norm(u), device=device)
        self.b = float(rng.uniform(-0.3, 0.3))

    def __call__(self, X):
        t = torch()
        r2 = ((X[:, None, :] - self.c[None]) ** 2).sum(-1)
        return (self.a * t.exp(-r2 / (2.0 * self.w ** 2))).sum(1) + t.tanh(8.0 * (X @ self.u - self.b))


def _target_numpy(job: SurrogateJob):
    """The job's target as a host function (the same parameters as _Target)."""

    rng = np.random.default_rng([job.seed, 7])
    d = job.dim
    c = rng.uniform(-1, 1, (8, d))
    w = rng.uniform(0.1, 0.6, 8) * np.sqrt(d / 2.0)
    a = rng.normal(size=8)
    u = rng.normal(size=d)
    u = u / np.linalg.norm(u)
    b = float(rng.uniform(-0.3, 0.3))

    def f(X):
        X = np.atleast_2d(X)
        r2 = ((X[:, None, :] - c[None]) ** 2).sum(-1)
        return (a * np.exp(-r2 / (2.0 * w ** 2))).sum(1) + np.tanh(8.0 * (X @ u - b))

    return f


def _ranges(starts, lens) -> np.ndarray:
    """The concatenation of arange(s, s + l) over (starts, lens)."""
    lens = np.asarray(lens, dtype=np.int64)
    return np.repeat(np.asarray(starts, dtype=np.int64) - (np.cumsum(lens) - lens), lens) + np.arange(int(lens.sum()))


def _runs(work):
    """(job state, node row starts, node row counts) for each job's consecutive nodes of ``work``."""
    out = []
    q0 = 0
    while q0 < len(work):
        st = work[q0][0]
        q1 = q0
        while q1 + 1 < len(work) and work[q1 + 1][0] is st:
            q1 += 1
        nodes = [nd for _, nd in work[q0:q1 + 1]]
        out.append((st, np.array([nd.r0 for nd in nodes], dtype=np.int64),
                    np.array([nd.r1 - nd.r0 for nd in nodes], dtype=np.int64)))
        q0 = q1 + 1
    return out


@dataclass
class _Node:
    path: str
    depth: int
    r0: int
    r1: int
    rows: list = field(default_factory=list)   # oblique constraints (a, b): a . x <= b
    coef: np.ndarray | None = None
    error: float = float("nan")
    theta: np.ndarray | None = None            # set when split


@dataclass
class JobResult:
    job_id: int
    arrival: float
    admitted: float
    finished: float
    n_rows: int
    leaves: list          # [(path, coef, error, r0, r1)] sorted by path
    splits: list          # [(path, theta)] sorted by path

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class _JobState:
    def __init__(self, job: SurrogateJob, device, admitted: float):
        t = torch()
        self.job = job
        self.admitted = admitted
        self.target = _Target(job, device)
        g = t.Generator(device=device)
        g.manual_seed(_key(job.seed, "x0") & ((1 << 63) - 1))
        cap = job.n_final
        self.X = t.empty((cap, job.dim), dtype=t.float64, device=device)
        self.y = t.empty(cap, dtype=t.float64, device=device)
        n0 = job.n_initial
        self.X[:n0] = t.rand((n0, job.dim), generator=g, dtype=t.float64, device=device) * 2.0 - 1.0
        self.y[:n0] = self.target(self.X[:n0])
        self.n = n0
        self.frontier = [_Node("r", 0, 0, n0)]
        self.leaves: list[_Node] = []
        self.splits: list[_Node] = []
        self.round = 0
        p = job.n_features
        self.min_side = job.min_side_points or 2 * p

    def done(self) -> bool:
        return not self.frontier and self.round >= self.job.rounds


class ServingEngine:
    """Admit, co-batch and complete surrogate-build jobs on one GPU.

    ``precision`` is the leaf-fit form ("mixed" or "fp64"); ``hbm_budget``
    bounds the summed footprint of admitted jobs and ``max_active`` their
    number.  ``run(jobs)`` replays arrivals against the wall clock (jobs are
    admitted no earlier than their arrival time) and returns one
    ``JobResult`` per job.

    The defaults are sized for one B200 (180 GB of HBM): 128 active jobs
    within 96 GB.  On the 2,000-job stream at 20 jobs/s, 64 / 128 / 256
    active jobs served 5.4 / 7.6 / 8.1 builds/s with p99 latencies of
    27.8 / 27.5 / 34.4 s: more jobs per tick fill the split launches, and
    past 128 the longer ticks raise latency more than throughput.
    """

    def __init__(self, precision: str = "mixed", hbm_budget: int = 96 << 30, max_active: int = 128,
                 stream=None):
        if precision not in ("mixed", "fp64"):
            raise ValueError("precision must be 'mixed' or 'fp64'")
        self.precision = precision
        self.hbm_budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.stream = stream
        self.ticks = 0
        self.peak_active = 0

    # ------------------------------------------------------------ public
    def run(self, jobs: list[SurrogateJob], clock=None, admit_until: float | None = None) -> list[JobResult]:
        """Serve ``jobs`` against the clock.  With ``admit_until`` (seconds),
        no job is admitted after that time: the admitted ones finish, and the
        rest are left unserved (``self.backlog`` counts those that had
        arrived by the end, ``self.unserved`` all of them)."""
        t = torch()
        dev = require_cuda()
        N.load_library()
        clock = clock or time.perf_counter
        pending = sorted(jobs, key=lambda j: (j.arrival, j.job_id))
        for j in pending:
            if job_footprint(j) > self.hbm_budget:
                raise ValueError(f"job {j.job_id} needs {job_footprint(j)} bytes, above the HBM budget")
        active: list[_JobState] = []
        results: list[JobResult] = []
        start = clock()
        used = 0
        self.backlog = self.unserved = 0
        while pending or active:
            now = clock() - start
            if admit_until is not None and now > admit_until and pending:
                if not active:
                    break
                pending_closed = True
            else:
                pending_closed = False
            while (not pending_closed and pending and pending[0].arrival <= now and len(active) < self.max_active
                   and used + job_footprint(pending[0]) <= self.hbm_budget):
                j = pending.pop(0)
                active.append(_JobState(j, dev, now))
                used += job_footprint(j)
            self.peak_active = max(self.peak_active, len(active))
            if not active:
                if pending_closed:
                    break
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
                continue
            self.tick(active)
            now = clock() - start
            for st in [s for s in active if s.done()]:
                active.remove(st)
                used -= job_footprint(st.job)
                results.append(self._result(st, now))
        t.cuda.synchronize()
        end = clock() - start
        self.unserved = len(pending)
        self.backlog = sum(1 for j in pending if j.arrival <= end)
        return sorted(results, key=lambda r: r.job_id)

    def build_alone(self, job: SurrogateJob) -> JobResult:
        """One job with nothing else on the device (the reference point of the
        alone-vs-mixed check)."""
        return self.run([SurrogateJob(**{**job.__dict__, "arrival": 0.0})])[0]

    # ------------------------------------------------------------ one tick
    def tick(self, active: list[_JobState]) -> None:
        self.ticks += 1
        due = [st for st in active if not st.frontier and st.round < st.job.rounds]
        if due:
            self._refine_all(due)
        work = [(st, nd) for st in active for nd in st.frontier]
        for st in active:
            st.frontier = []
        if not work:
            return
        self._fit_and_split(work)

    def _gather(self, work):
        """Concatenate the rows of the given (job, node) pairs into one batch."""

        t = torch()
        xs, ys = [], []
        for st, r0s, lens in _runs(work):
            if np.all(r0s[1:] == r0s[:-1] + lens[:-1]):  # one contiguous range of the job's rows
                a, b = int(r0s[0]), int(r0s[0] + lens.sum())
                xs.append(st.X[a:b].reshape(-1))
                ys.append(st.y[a:b])
            else:
                idx = t.as_tensor(_ranges(r0s, lens), device=st.X.device)
                xs.append(st.X[idx].reshape(-1))
                ys.append(st.y[idx])
        n = np.array([nd.r1 - nd.r0 for _, nd in work], dtype=np.int64)
        d = np.array([st.job.dim for st, _ in work], dtype=np.int32)
        ro = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
        xo = np.concatenate([[0], np.cumsum(n * d)])[:-1].astype(np.int64)
        return t.cat(xs), t.cat(ys), ro, xo, d

    def _fit_and_split(self, work) -> None:
        t = torch()
        x, y, ro, xo, d = self._gather(work)
        kinds = np.array([st.job.kind for st, _ in work], dtype=np.int32)
        ridge = np.array([st.job.ridge for st, _ in work])
        pmax = max(st.job.n_features for st, _ in work)
        fit = solve_weighted_ridge_batched(x, y, None, ro, d, kinds, ridge, x_offsets=xo, precision=self.precision,
                                           max_features=pmax, max_dim=int(d.max()), weight_floor=0.0,
                                           stream=self.stream)
        sse, ssy = segment_residuals(x, y, ro, d, kinds, fit.beta, x_offsets=xo, stream=self.stream)
        beta = fit.beta.cpu().numpy()
        status = fit.status.cpu().numpy()
        err = np.sqrt(sse.cpu().numpy() / np.maximum(ssy.cpu().numpy(), 1e-300))
        split_idx = []
        for k, (st, nd) in enumerate(work):
            p = st.job.n_features
            nd.coef = beta[k, :p].copy()
            nd.error = float(err[k]) if status[k] == 0 else float("inf")
            n = nd.r1 - nd.r0
            if (status[k] == 0 and nd.error <= st.job.error_threshold) or nd.depth >= st.job.max_depth \
                    or n < 2 * st.min_side:
                st.leaves.append(nd)
            else:
                split_idx.append(k)
        # (The CTA form runs two CTAs per SM here: many small single-restart
        # nodes keep one CTA per SM waiting at its barriers; 1.34x on a level
        # of 4,609 such d = 32 nodes.)
        # max_iters is a per-call parameter of the split search (one call per
        # distinct value); the minimum side count goes per node, so nodes of
        # every dimension share a launch.  Nodes for the warp-per-restart form
        # (d and p at most 23, at most WARP_MAX_ROWS rows: larger nodes take
        # the CTA form, whose gangs span many SMs) and the others go to
        # separate launches, since the form of a launch is one for all its
        # nodes: so a node's split never depends on the nodes batched with it.
        groups: dict[tuple[int, bool], list[int]] = {}
        for k in split_idx:
            job = work[k][0].job
            warp = (job.dim <= WARP_MAX_DIM and job.n_features <= WARP_MAX_FEATURES
                    and ro[k + 1] - ro[k] <= WARP_MAX_ROWS)
            groups.setdefault((job.max_iters, warp), []).append(k)
        for (iters, warp), ks in sorted(groups.items()):
            self._split([work[k] for k in ks], x, y, ro, xo, d, kinds, ks, iters, warp)

    def _split(self, sub, x, y, ro, xo, d, kinds, idx, iters, warp) -> None:
        t = torch()
        dev = x.device
        # the split nodes' rows, gathered from the fit batch: a job's nodes are
        # consecutive there, with one row width, so one slice or gather per job
        xl, yl = [], []
        q0 = 0
        while q0 < len(idx):
            q1 = q0
            while q1 + 1 < len(idx) and sub[q1 + 1][0] is sub[q0][0]:
                q1 += 1
            ks = np.asarray(idx[q0:q1 + 1])
            dim = int(d[ks[0]])
            lens = ro[ks + 1] - ro[ks]
            if np.all(ks[1:] == ks[:-1] + 1):
                a, b = int(ro[ks[0]]), int(ro[ks[-1] + 1])
                xl.append(x[int(xo[ks[0]]): int(xo[ks[0]]) + (b - a) * dim])
                yl.append(y[a:b])
            else:
                rows = t.as_tensor(_ranges(ro[ks], lens), device=dev)
                base = int(xo[ks[0]]) - int(ro[ks[0]]) * dim   # the job's block of x, viewed as rows
                blk = x[base + int(ro[ks[0]]) * dim: base + int(ro[ks[-1] + 1]) * dim].view(-1, dim)
                xl.append(blk[rows - int(ro[ks[0]])].reshape(-1))
                yl.append(y[rows])
            q0 = q1 + 1
        xs = t.cat(xl)
        ys = t.cat(yl)
        n = np.array([ro[k + 1] - ro[k] for k in idx], dtype=np.int64)
        dd = d[idx]
        sro = np.concatenate([[0], np.cumsum(n)]).astype(np.int64)
        sxo = np.concatenate([[0], np.cumsum(n * dd)])[:-1].astype(np.int64)
        keys = np.array([_key(st.job.seed, "split", nd.path) for st, nd in sub], dtype=np.uint64)
        temps = np.array([st.job.temperature for st, _ in sub])
        ridge = np.array([st.job.ridge for st, _ in sub])
        min_side = np.array([st.min_side for st, _ in sub], dtype=np.int32)
        sp = SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 1.0, max_iters=iters, grad_atol=1e-8,
                                 grad_rtol=1e-5, min_side_points=int(min_side.min()), min_side_fraction=0.0,
                                 n_restarts=1)
        res = split_level(sp, xs, ys, sro, dd, kinds[idx], temps, ridge, x_offsets=sxo, hard_refit=False,
                          node_keys=keys, max_dim=int(dd.max()), max_features=int(max(st.job.n_features for st, _ in sub)),
                          min_side_points=min_side, group_restarts=0, trial_steps=0,
                          ctas_per_sm=0 if warp else 2, restart_warps=int(warp), stream=self.stream)
        failure = res.failure.cpu().numpy()
        theta = res.theta
        ok = failure == 0
        split_flag = t.as_tensor(ok.astype(np.int8), device=dev)
        perm = t.empty(int(sro[-1]), dtype=t.int64, device=dev)
        n_right = t.empty(len(sub), dtype=t.int32, device=dev)
        lib = N.load_library()
        ro_t = t.as_tensor(sro, device=dev)
        xo_t = t.as_tensor(sxo, device=dev)
        d_t = t.as_tensor(dd, device=dev)
        k_t = t.as_tensor(kinds[idx], device=dev)
        seg = N.ArtSegments(len(sub), ptr(ro_t), ptr(xo_t), ptr(d_t), ptr(k_t))
        N.check(lib.art_partition_rows(C.byref(seg), ptr(xs), ptr(theta), int(theta.shape[1]), ptr(split_flag),
                                       ptr(perm), ptr(n_right), stream_handle(self.stream)), "art_partition_rows")
        nr = n_right.cpu().numpy()
        th = theta.cpu().numpy()
        # each job's nodes are consecutive in the batch, with one row width:
        # its rows in partitioned order by one gather, written back by one
        # slice copy (or one indexed copy when its nodes' row ranges have gaps);
        # unsplit nodes are copied unchanged
        j0 = 0
        while j0 < len(sub):
            st = sub[j0][0]
            j1 = j0
            while j1 + 1 < len(sub) and sub[j1 + 1][0] is st:
                j1 += 1
            dim = st.job.dim
            s0, s1 = int(sro[j0]), int(sro[j1 + 1])
            src = xs[int(sxo[j0]): int(sxo[j0]) + (s1 - s0) * dim].view(s1 - s0, dim)
            loc = perm[s0:s1] - s0
            r0s = np.array([sub[j][1].r0 for j in range(j0, j1 + 1)], dtype=np.int64)
            lens = n[j0:j1 + 1]
            if np.all(r0s[1:] == r0s[:-1] + lens[:-1]):
                st.X[int(r0s[0]): int(r0s[0]) + s1 - s0] = src[loc]
                st.y[int(r0s[0]): int(r0s[0]) + s1 - s0] = ys[s0:s1][loc]
            else:
                dst = t.as_tensor(np.repeat(r0s - (np.cumsum(lens) - lens), lens) + np.arange(s1 - s0), device=dev)
                st.X[dst] = src[loc]
                st.y[dst] = ys[s0:s1][loc]
            j0 = j1 + 1
        for j, (st, nd) in enumerate(sub):
            if not ok[j]:
                st.leaves.append(nd)   # no valid split: the node stays a leaf
                continue
            a, b = int(sro[j]), int(sro[j + 1])
            dim = st.job.dim
            nl = (b - a) - int(nr[j])
            w, z = th[j, :dim].copy(), float(th[j, dim])
            nd.theta = th[j, : dim + 1].copy()
            st.splits.append(nd)
            st.frontier.append(_Node(nd.path + "L", nd.depth + 1, nd.r0, nd.r0 + nl, nd.rows + [(w, z)]))
            st.frontier.append(_Node(nd.path + "R", nd.depth + 1, nd.r0 + nl, nd.r1, nd.rows + [(-w, -z)]))

    # ------------------------------------------------------------ rounds
    _CHAINS = 8            # fewest chains per refined leaf
    _MAX_CHAINS = 256      # most chains per refined leaf
    _PER_CHAIN = 128       # target samples per chain

    def _refine_all(self, states: list[_JobState]) -> None:
        """One adaptive round for every given job: grow_fraction * n0 new
        hit-and-run samples inside the leaves with the largest fit error, one
        ``art_hit_and_run`` call per input dimension for all jobs together."""

        from .sampling import DevicePolytopes, hit_and_run_device

        t = torch()
        plans = []
        for st in states:
            job = st.job
            st.round += 1
            leaves = sorted(st.leaves, key=lambda nd: (-nd.error, nd.path))[: job.refine_leaves]
            if not leaves:
                continue
            total = int(round(job.grow_fraction * job.n_initial))
            per = [total // len(leaves) + (1 if i < total % len(leaves) else 0) for i in range(len(leaves))]
            plans.append((st, leaves, per))
        by_dim: dict[int, list] = {}
        for plan in plans:
            by_dim.setdefault(plan[0].job.dim, []).append(plan)
        for dim, group in sorted(by_dim.items()):
            leaves_all = [(st, nd, per[i]) for st, leaves, per in group for i, nd in enumerate(leaves)]
            # a leaf's samples come from several short chains (one long chain
            # is a sequential walk of n * thinning steps); each chain starts at
            # the leaf's sample mean and burns in 20 + 2 d steps
            chains = [int(min(self._MAX_CHAINS, max(self._CHAINS, -(-n // self._PER_CHAIN))))
                      for _, _, n in leaves_all]
            dev = group[0][0].X.device
            m = len(leaves_all)
            A = [np.asarray(w, float) for _, nd, _ in leaves_all for w, _ in nd.rows]
            bb = [float(z) for _, nd, _ in leaves_all for _, z in nd.rows]
            rof = np.concatenate([[0], np.cumsum([len(nd.rows) for _, nd, _ in leaves_all])]).astype(np.int64)
            polys = DevicePolytopes(
                dim, t.full((m, dim), -1.0, dtype=t.float64, device=dev), t.full((m, dim), 1.0, dtype=t.float64, device=dev),
                t.as_tensor(rof, device=dev),
                t.as_tensor(np.array(A).reshape(-1, dim) if A else np.zeros((1, dim)), device=dev),
                t.as_tensor(np.array(bb) if bb else np.zeros(1), device=dev), max(1, int(np.diff(rof).max())))
            # start every chain at its leaf's sample mean (inside the convex leaf)
            means = t.stack([st.X[nd.r0:nd.r1].mean(0) for st, nd, _ in leaves_all])
            cnt = t.as_tensor(np.asarray(chains), device=dev)
            x0 = means.repeat_interleave(cnt, 0)
            cpoly = np.repeat(np.arange(m, dtype=np.int32), chains)
            seeds = np.array([_key(st.job.seed, "har", st.round, nd.path, c) for (st, nd, _), ch in
                              zip(leaves_all, chains) for c in range(ch)], dtype=np.uint64)
            n_rounds = max(1, max(-(-n // ch) for (_, _, n), ch in zip(leaves_all, chains)))
            samples, _, status = hit_and_run_device(polys, cpoly, x0, burn_in=20 + 2 * dim, thinning=10,
                                                    n_rounds=n_rounds, seeds=seeds, stream=self.stream)
            first = np.concatenate([[0], np.cumsum(chains)])
            for i, (st, nd, n) in enumerate(leaves_all):
                nd._new = samples[:, first[i]:first[i + 1], :].reshape(-1, dim)[:n]
        for st, leaves, _ in plans:
            self._reopen(st, {nd.path for nd in leaves})

    def _reopen(self, st: _JobState, paths: set) -> None:
        """Rebuild the node-sorted layout: every leaf keeps its rows, the
        reopened ones get their new rows appended and return to the frontier."""

        t = torch()
        order = sorted(st.leaves, key=lambda nd: nd.r0)
        Xn, yn, r = [], [], 0
        st.leaves = []
        for nd in order:
            rows_x = st.X[nd.r0:nd.r1]
            rows_y = st.y[nd.r0:nd.r1]
            if nd.path in paths:
                xn = nd._new
                rows_x = t.cat([rows_x, xn])
                rows_y = t.cat([rows_y, st.target(xn)])
                del nd._new
            cnt = rows_x.shape[0]
            Xn.append(rows_x)
            yn.append(rows_y)
            nd.r0, nd.r1 = r, r + cnt
            r += cnt
            (st.frontier if nd.path in paths else st.leaves).append(nd)
        X = t.cat(Xn)
        y = t.cat(yn)
        st.X[:r] = X
        st.y[:r] = y
        st.n = r

    def _result(self, st: _JobState, now: float) -> JobResult:
        leaves = sorted(((nd.path, nd.coef, nd.error, nd.r0, nd.r1) for nd in st.leaves), key=lambda v: v[0])
        splits = sorted(((nd.path, nd.theta) for nd in st.splits), key=lambda v: v[0])
        return JobResult(st.job.job_id, st.job.arrival, st.admitted, now, st.n, leaves, splits)
