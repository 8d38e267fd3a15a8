"""Temperature scale on the GPU: the batched median nearest-neighbour distance
(art_median_nn_distance) against the reference's kd-tree query and the numpy
brute force, alone and through estimate_temperature with the reference's
subsampling (tolerance 1e-13 relative: the distances differ at most in the
summation order of the squared coordinates)."""

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def brute_median_nn(X):
    D = np.linalg.norm(X[:, None, :] - X[None, :, :], axis=2)
    np.fill_diagonal(D, np.inf)
    return float(np.median(D.min(axis=1)))


def test_batched_median_nn_matches_kdtree_and_brute_force():
    from scipy.spatial import cKDTree

    from art.temperature import median_nn_distance_batched

    rng = np.random.default_rng(12)
    sets = []
    for m, d in [(2, 1), (3, 2), (17, 8), (512, 2), (512, 20), (1000, 64), (301, 5), (64, 3)]:
        X = rng.normal(size=(m, d)) * rng.uniform(0.1, 3.0, d)
        sets.append(X)
    dup = rng.uniform(-1, 1, (40, 4))
    sets.append(np.vstack([dup, dup[:7]]))            # duplicated points: distance 0 neighbours
    out = median_nn_distance_batched(sets, c=0.37).cpu().numpy()
    for X, v in zip(sets, out):
        ref_kd = float(np.median(cKDTree(X).query(X, k=2)[0][:, 1]))
        np.testing.assert_allclose(v, 0.37 * ref_kd, rtol=1e-13, atol=0.0)
        np.testing.assert_allclose(v, 0.37 * brute_median_nn(X), rtol=1e-13, atol=0.0)


def test_small_sets_and_limits():
    from art import _native as N
    from art.temperature import median_nn_distance_batched

    out = median_nn_distance_batched([np.zeros((1, 3)), np.array([[0.0], [2.0]])]).cpu().numpy()
    assert np.isnan(out[0]) and out[1] == 2.0
    with pytest.raises(ValueError):
        median_nn_distance_batched([np.zeros((N.MEDIAN_NN_MAX_SET + 1, 2))])
    with pytest.raises(ValueError):
        median_nn_distance_batched([np.zeros((4, 2))], c=0.0)


@pytest.mark.parametrize("d", [2, 9, 30])
def test_estimate_temperature_device_equals_kdtree(d):
    from art.temperature import estimate_temperature

    rng = np.random.default_rng(40 + d)
    X = rng.uniform(-1, 1, (3000, d))
    for seed in (1, 2):
        t_kd = estimate_temperature(X, "median_nn", c=0.1, max_points=512, random_state=seed, nn_method="kdtree")
        t_dev = estimate_temperature(X, "median_nn", c=0.1, max_points=512, random_state=seed, nn_method="device")
        np.testing.assert_allclose(t_dev, t_kd, rtol=1e-13, atol=0.0)


def test_max_set_below_a_set_size_gives_nan_for_that_set_only():
    """A C caller that passes max_set smaller than one of its sets: that set
    gets NaN (it is not processed, so the shared arrays sized by max_set are
    never overrun) and the other sets are unaffected.  The inputs are valid
    device buffers; only the size bound is too small."""
    import torch

    from art import _native as N
    from art._device import ptr

    rng = np.random.default_rng(7)
    sets = [rng.uniform(-1, 1, (40, 3)), rng.uniform(-1, 1, (300, 3)), rng.uniform(-1, 1, (12, 3))]
    sizes = np.array([len(P) for P in sets], np.int64)
    dev = torch.device("cuda", 0)
    x = torch.tensor(np.concatenate([P.reshape(-1) for P in sets]), dtype=torch.float64, device=dev)
    xo = torch.tensor(np.r_[0, np.cumsum(sizes * 3)[:-1]], dtype=torch.int64, device=dev)
    dims = torch.full((3,), 3, dtype=torch.int32, device=dev)
    so = torch.tensor(np.r_[0, np.cumsum(sizes)], dtype=torch.int64, device=dev)
    rows = torch.tensor(np.concatenate([np.arange(m) for m in sizes]), dtype=torch.int64, device=dev)
    out = torch.full((3,), -1.0, dtype=torch.float64, device=dev)
    lib = N.load_library()
    rc = lib.art_median_nn_distance(3, ptr(x), ptr(xo), ptr(dims), ptr(so), ptr(rows), 64, 1.0, ptr(out), None)
    assert rc == 0
    got = out.cpu().numpy()
    assert np.isnan(got[1])
    np.testing.assert_allclose(got[0], brute_median_nn(sets[0]), rtol=1e-13, atol=0.0)
    np.testing.assert_allclose(got[2], brute_median_nn(sets[2]), rtol=1e-13, atol=0.0)
