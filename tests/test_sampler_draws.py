"""Batched sampler classes with rng_mode="reference": the host side draws the
directions and chord uniforms in the reference's order and layout
(BatchedHitAndRunSampler / NumbaBatchedHitAndRunSampler step-major,
ParallelNumbaBatchedHitAndRunSampler chain-major with per-worker SFC64
blocks, the tail round for a partial last round, covariance shaping).

CPU part: those host draws, run through the oracle's chain restatement,
reproduce the reference classes' own samples (fixtures made by the reference,
tests/golden/make_golden.py sampler) to 1e-12.  GPU part: the public
``sample`` call (draws injected into art_hit_and_run) reproduces them too."""

import ast

import numpy as np
import pytest

from conftest import GOLDEN, gpu_available
from oracle import sampling as H

G = np.load(GOLDEN / "har_sampler_golden.npz")


def _case(i):
    seed, cls, d, k, n, kw, x0kind = ast.literal_eval(str(G[f"m{i}_spec"]))
    extra = dict(kw)
    if f"m{i}_vecs" in G.files:
        extra.update(direction_eigenvectors=G[f"m{i}_vecs"], direction_eigenvalues=G[f"m{i}_vals"])
    pool = G[f"m{i}_pool"]
    x0 = None if x0kind == "none" else (pool[0] if x0kind == "point" else pool)
    return seed, cls, d, n, extra, x0


def _sampler(cls, extra):
    import art

    return getattr(art, cls)(rng_mode="reference", **extra)


@pytest.mark.parametrize("i", range(int(G["count"])))
def test_host_draws_with_oracle_chains_reproduce_reference_sampler(i):
    from art.domain import PolytopeRegion
    from art.sampling import as_rng

    seed, cls, d, n, extra, x0 = _case(i)
    A, b = G[f"m{i}_A"], G[f"m{i}_b"]
    s = _sampler(cls, extra)
    region = PolytopeRegion(A, b)
    rng = as_rng(seed + 7)
    C = min(s.n_chains, n)
    points = s._initial_points(region, C, rng, x0)
    stride = max(1, s.thinning)
    full, rem = divmod(n, C)
    dirs, unif = s._reference_draws(rng, C, s.burn_in + full * stride, d)
    out, last = H.chains_batched(A, b, points, dirs, unif, s.burn_in, stride, full)
    got = [out.reshape(-1, d)]
    if rem:
        td, tu = s._reference_draws(rng, rem, stride, d)
        extra_rows, _ = H.chains_batched(A, b, last[:rem], td, tu, 0, stride, 1)
        got.append(extra_rows.reshape(-1, d))
    np.testing.assert_allclose(np.concatenate(got)[:n], G[f"m{i}_samples"], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("i", range(int(G["count"])))
def test_public_batched_sampler_reference_mode_equals_reference(i):
    from art.domain import PolytopeRegion

    seed, cls, d, n, extra, x0 = _case(i)
    s = _sampler(cls, extra)
    got = s.sample(PolytopeRegion(G[f"m{i}_A"], G[f"m{i}_b"]), n, random_state=seed + 7, x0=x0)
    np.testing.assert_allclose(got, G[f"m{i}_samples"], rtol=1e-12, atol=1e-12)
