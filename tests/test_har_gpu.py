"""Hit-and-run on the GPU: injected-draw parity with the reference (golden
fixtures from its numba kernel and scalar sampler, tolerance 1e-12), and
statistical checks of the device-RNG chains (feasibility, KS uniformity
against an exact rejection sample, lag autocorrelation decay)."""

import numpy as np
import pytest

from conftest import GOLDEN, gpu_available
from oracle import sampling as H

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

G = np.load(GOLDEN / "har_golden.npz") if (GOLDEN / "har_golden.npz").exists() else None


def box(d):
    return -np.ones(d), np.ones(d)


@pytest.mark.parametrize("i", range(4))
def test_batched_chains_match_reference_numba_with_injected_draws(i):
    from art.sampling import device_polytopes, hit_and_run_device

    d, k, C, burn, thin, rounds = (int(v) for v in G[f"b{i}_meta"])
    Ao, bo, x0 = G[f"b{i}_Ao"], G[f"b{i}_bo"], G[f"b{i}_x0"]
    Ab, bb = H.box_rows(*box(d))
    polys = device_polytopes([(np.vstack([Ab, Ao]), np.concatenate([bb, bo]))])
    samples, last, status = hit_and_run_device(
        polys, np.zeros(C, np.int32), x0, burn_in=burn, thinning=thin, n_rounds=rounds,
        mode="batched", directions=G[f"b{i}_dirs"], uniforms=G[f"b{i}_unif"])
    assert (status.cpu().numpy() == 0).all()
    np.testing.assert_allclose(samples.cpu().numpy(), G[f"b{i}_samples"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("i", range(3))
def test_scalar_chain_matches_reference_sampler_with_injected_draws(i):
    from art.sampling import device_polytopes, hit_and_run_device

    d, k, burn, thin, n = (int(v) for v in G[f"s{i}_meta"])
    Ao, bo, x0 = G[f"s{i}_Ao"], G[f"s{i}_bo"], G[f"s{i}_x0"]
    Ab, bb = H.box_rows(*box(d))
    polys = device_polytopes([(np.vstack([Ab, Ao]), np.concatenate([bb, bo]))])
    samples, _, status = hit_and_run_device(
        polys, [0], x0[None, :], burn_in=burn, thinning=thin, n_rounds=n, mode="scalar",
        directions=G[f"s{i}_dirs"][None], uniforms=G[f"s{i}_unif"][None])
    assert int(status.cpu().numpy()[0]) == 0
    np.testing.assert_allclose(samples.cpu().numpy()[:, 0, :], G[f"s{i}_samples"], rtol=1e-12, atol=1e-12)


def test_public_sampler_reference_rng_mode_equals_reference_chain():
    """HitAndRunSampler(rng_mode='reference') consumes the generator like the reference."""
    from art.domain import PolytopeRegion
    from art.sampling import HitAndRunSampler

    rng = np.random.default_rng(31)
    d = 3
    Ab, bb = H.box_rows(*box(d))
    a = rng.normal(size=d)
    a /= np.linalg.norm(a)
    A = np.vstack([Ab, a])
    b = np.concatenate([bb, [0.3]])
    x0 = np.zeros(d)
    region = PolytopeRegion(A, b)
    out = HitAndRunSampler(burn_in=4, thinning=3, rng_mode="reference").sample(region, 25, random_state=77, x0=x0)
    # replay the same generator calls on the host
    g = np.random.default_rng(77)
    steps = 4 + 25 * 3
    dirs, unif = [], []
    for _ in range(steps):
        dirs.append(g.normal(size=d))
        unif.append(g.uniform(0.0, 1.0))
    ref = H.chain_scalar(A, b, x0, np.array(dirs), np.array(unif), 4, 3, 25)
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-12)


def c4_polytopes(rng, d, count):
    regs, starts = [], []
    for _ in range(count):
        k = int(rng.integers(4, 13))
        c = rng.uniform(-0.5, 0.5, d)
        A = rng.normal(size=(k, d))
        A /= np.linalg.norm(A, axis=1, keepdims=True)
        b = A @ c + rng.uniform(0.05, 0.5, k)
        Ab, bb = H.box_rows(*box(d))
        regs.append((np.vstack([Ab, A]), np.concatenate([bb, b])))
        starts.append(c)
    return regs, np.array(starts)


@pytest.mark.parametrize("d", [2, 8, 16, 32, 64])
def test_device_chains_stay_feasible(d):
    from art.sampling import device_polytopes, hit_and_run_device

    rng = np.random.default_rng(40 + d)
    regs, starts = c4_polytopes(rng, d, 64)
    polys = device_polytopes(regs)
    C = 256
    cp = np.arange(C) % 64
    samples, last, status = hit_and_run_device(polys, cp, starts[cp], burn_in=0, thinning=10, n_rounds=20,
                                               mode="batched", seeds=np.arange(C) + 1000 * d)
    assert (status.cpu().numpy() == 0).all()
    S = samples.cpu().numpy()
    for c in range(C):
        A, b = regs[cp[c]]
        assert np.all(S[:, c, :] @ A.T <= b + 1e-9)
    # chains move and differ
    assert np.std(S[-1, :, 0]) > 0


def test_device_chains_are_uniform_ks_and_decorrelate():
    from scipy.stats import ks_2samp

    from art.sampling import device_polytopes, hit_and_run_device

    rng = np.random.default_rng(5)
    d = 2
    a = np.array([1.0, 1.0]) / np.sqrt(2)
    A = np.vstack([H.box_rows(*box(d))[0], a])
    b = np.concatenate([H.box_rows(*box(d))[1], [0.4]])
    polys = device_polytopes([(A, b)])
    C = 4096
    x0 = np.zeros((C, d))
    samples, _, status = hit_and_run_device(polys, np.zeros(C, np.int32), x0, burn_in=200, thinning=10,
                                            n_rounds=50, mode="batched", seeds=np.arange(C) * 7919 + 3)
    S = samples.cpu().numpy()
    exact = H.rejection_sample(A[-1:], b[-1:], -np.ones(d), np.ones(d), 50000, rng)
    flat = S.reshape(-1, d)
    for j in range(d):
        assert ks_2samp(flat[::7, j], exact[:, j]).pvalue > 1e-3
    proj = S[:, :, 0] + 0.5 * S[:, :, 1]      # (rounds, chains): thinned series per chain
    acf = H.autocorrelation_by_lag(proj, [1, 5, 20])
    assert np.median(acf[2]) < 0.2


def test_device_rng_is_deterministic_and_counter_advances():
    from art.sampling import device_polytopes, hit_and_run_device

    d = 4
    Ab, bb = H.box_rows(*box(d))
    polys = device_polytopes([(Ab, bb)])
    x0 = np.zeros((8, d))
    kw = dict(burn_in=0, thinning=3, n_rounds=5, mode="batched", seeds=np.arange(8) + 11)
    a = hit_and_run_device(polys, np.zeros(8, np.int32), x0, **kw)[0].cpu().numpy()
    b = hit_and_run_device(polys, np.zeros(8, np.int32), x0, **kw)[0].cpu().numpy()
    c = hit_and_run_device(polys, np.zeros(8, np.int32), x0, counter_base=1000, **kw)[0].cpu().numpy()
    np.testing.assert_array_equal(a, b)
    assert not np.allclose(a, c)


def test_infeasible_start_and_empty_chord_are_reported():
    from art.sampling import device_polytopes, hit_and_run_device

    d = 2
    Ab, bb = H.box_rows(*box(d))
    polys = device_polytopes([(Ab, bb)])
    _, _, status = hit_and_run_device(polys, [0, 0], np.array([[0.0, 0.0], [3.0, 0.0]]), burn_in=0,
                                      thinning=1, n_rounds=2, mode="batched", seeds=[1, 2])
    st = status.cpu().numpy()
    assert st[0] == 0 and st[1] == 2


def test_device_draws_with_covariance_shaped_directions():
    """Device draws with a direction spectrum move along u = Q diag(sqrt(l)) z:
    chains stay feasible and their sample covariance is elongated along the
    leading eigenvector, as the reference's covariance-shaped sampler is."""

    from art.domain import BoxDomain
    from art.sampling import HitAndRunSampler

    region = BoxDomain.hypercube(2, -1.0, 1.0).as_region()
    th = np.pi / 6
    Q = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    vals = np.array([1.0, 1e-4])
    iso = HitAndRunSampler(burn_in=50, thinning=1, rng_mode="device")
    aniso = HitAndRunSampler(burn_in=50, thinning=1, rng_mode="device", direction_eigenvectors=Q,
                             direction_eigenvalues=vals)
    X = aniso.sample(region, 4000, random_state=3, x0=np.zeros(2))
    assert X.shape == (4000, 2) and np.all(region.contains(X))
    steps = np.diff(X, axis=0)
    steps = steps[np.linalg.norm(steps, axis=1) > 0]
    ang = np.abs(steps @ Q[:, 1]) / np.linalg.norm(steps, axis=1)   # component along the small axis
    assert np.median(ang) < 0.05
    Y = iso.sample(region, 4000, random_state=3, x0=np.zeros(2))
    sy = np.diff(Y, axis=0)
    assert np.median(np.abs(sy @ Q[:, 1]) / np.linalg.norm(sy, axis=1)) > 0.3
    again = aniso.sample(region, 4000, random_state=3, x0=np.zeros(2))
    np.testing.assert_array_equal(X, again)


@pytest.mark.parametrize("d", [3, 8, 16, 32])
def test_chains_of_mixed_row_counts_share_warps_with_injected_draws(d):
    """Teams of one warp run polytopes of 0 to 16 oblique rows (the row loop
    stops at the warp's largest count; each lane bounds only its own rows):
    every chain equals the oracle's batched transition on the same draws."""
    from art.sampling import device_polytopes, hit_and_run_device

    rng = np.random.default_rng(70 + d)
    regs, starts = [], []
    for j in range(40):
        k = int(rng.integers(0, 17)) if j % 5 else 0
        c = rng.uniform(-0.5, 0.5, d)
        A = rng.normal(size=(k, d))
        A /= np.maximum(np.linalg.norm(A, axis=1, keepdims=True), 1e-12)
        b = A @ c + rng.uniform(0.05, 0.5, k)
        Ab, bb = H.box_rows(*box(d))
        regs.append((np.vstack([Ab, A]), np.concatenate([bb, b])))
        starts.append(c)
    C, steps = 96, 24
    cp = rng.permutation(np.arange(C) % len(regs)).astype(np.int32)
    x0 = np.array(starts)[cp]
    dirs, unif = rng.normal(size=(C, steps, d)), rng.uniform(size=(C, steps))
    samples, last, status = hit_and_run_device(device_polytopes(regs), cp, x0, burn_in=0, thinning=3,
                                               n_rounds=steps // 3, mode="batched", directions=dirs,
                                               uniforms=unif)
    assert (status.cpu().numpy() == 0).all()
    S = samples.cpu().numpy()
    for c in range(C):
        A, b = regs[cp[c]]
        ref, _ = H.chains_batched(A, b, x0[c:c + 1], dirs[c:c + 1], unif[c:c + 1], 0, 3, steps // 3)
        np.testing.assert_allclose(S[:, c, :], ref[:, 0, :], rtol=1e-12, atol=1e-12, err_msg=f"chain {c}")


def _rejection_in_chunks(A, b, d, n, rng, chunk=200_000):
    """Exactly uniform points of the polytope by rejection from the box, in chunks."""
    out, have = [], 0
    for _ in range(2000):
        X = rng.uniform(-1.0, 1.0, (chunk, d))
        keep = np.all(X @ A.T <= b[None, :], axis=1)
        out.append(X[keep])
        have += int(keep.sum())
        if have >= n:
            break
    return np.concatenate(out)[:n]


@pytest.mark.parametrize("d,k,seed", [(8, 12, 1), (8, 7, 2), (64, 4, 3), (64, 5, 4)])
def test_c4_polytope_chains_are_uniform_ks_and_decorrelate(d, k, seed):
    """The C4 sampling configuration (box [-1,1]^d cut by k oblique
    halfspaces with a Chebyshev ball of radius >= 0.05, directions uniform on
    the sphere, thinning 10, device Philox draws, FP64 chords): 2048 chains
    from the ball's centre, the last state of each after the burn-in is one
    independent draw; each coordinate passes a two-sample KS test against an
    exactly uniform rejection sample (p > 1e-4 for every coordinate), and the
    thinned series decorrelate (median autocorrelation below 0.2 at a lag of
    200 steps for d = 8 and 2,000 steps for d = 64).
    The burn-in is 2,000 steps at d = 8 and 20,000 at d = 64 (hit-and-run
    mixes in O(d^2) steps)."""
    from scipy.stats import ks_2samp

    from art.sampling import device_polytopes, hit_and_run_device

    rng = np.random.default_rng(900 + seed)
    c = rng.uniform(-0.5, 0.5, d)
    Ao = rng.normal(size=(k, d))
    Ao /= np.linalg.norm(Ao, axis=1, keepdims=True)
    bo = Ao @ c + rng.uniform(0.05, 0.5, k)
    assert min(np.min(bo - Ao @ c), np.min(1 - np.abs(c))) >= 0.05      # Chebyshev ball of radius 0.05
    Ab, bb = H.box_rows(*box(d))
    A, b = np.vstack([Ab, Ao]), np.concatenate([bb, bo])
    C = 2048
    burn = 2000 if d <= 8 else 20000
    polys = device_polytopes([(A, b)])
    last_round, _, status = hit_and_run_device(polys, np.zeros(C, np.int32), np.repeat(c[None], C, 0), burn_in=burn,
                                               thinning=10, n_rounds=1, mode="batched",
                                               seeds=np.arange(C, dtype=np.uint64) * 7919 + 11 * seed)
    assert (status.cpu().numpy() == 0).all()
    draws = last_round.cpu().numpy()[0]
    assert np.all(draws @ Ao.T <= bo + 1e-9) and np.all(np.abs(draws) <= 1 + 1e-12)
    exact = _rejection_in_chunks(Ao, bo, d, 4000, rng)
    pvals = [ks_2samp(draws[:, j], exact[:, j]).pvalue for j in range(d)]
    assert min(pvals) > 1e-4, min(pvals)
    # autocorrelation of the thinned series of 256 continued chains: it
    # decays, and is below 0.2 after 200 steps at d = 8 and 2,000 at d = 64
    rounds, lag = (200, 20) if d <= 8 else (1000, 200)
    series, _, status = hit_and_run_device(polys, np.zeros(256, np.int32), draws[:256], burn_in=0, thinning=10,
                                           n_rounds=rounds, mode="batched",
                                           seeds=np.arange(256, dtype=np.uint64) + 10_000 * seed)
    S = series.cpu().numpy()
    proj = S @ (np.ones(d) / np.sqrt(d))
    acf = H.autocorrelation_by_lag(proj, [1, lag])
    assert np.median(acf[1]) < 0.2 and np.median(acf[1]) < np.median(acf[0])
