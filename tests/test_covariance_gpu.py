"""Pilot-chain covariance spectra on the GPU (art_covariance_eigh) against the
host form the reference uses, sample_covariance_eigendecomposition
(sampling.py:86-106: covariance with n - 1, numpy.linalg.eigh).

Eigenvalues agree to 1e-12 of the largest; eigenvectors agree up to sign
where the eigenvalues are separated, reconstruct the covariance to 1e-12 and
are orthonormal to 1e-13; the sign rule (largest-magnitude component
positive) holds; degenerate inputs report their status."""

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("d", [1, 2, 3, 8, 16, 33, 64])
def test_batched_spectra_match_numpy_eigh(d):
    from art.sampling import covariance_eigendecomposition_batched, sample_covariance_eigendecomposition

    rng = np.random.default_rng(100 + d)
    sets = []
    for n in (2, 7, 40, 5 * d + 3, 300):
        scale = np.exp(rng.uniform(-3, 3, d))                 # condition numbers up to ~e^12
        Q, _ = np.linalg.qr(rng.normal(size=(d, d)))
        sets.append((rng.normal(size=(n, d)) * scale) @ Q.T + rng.normal(size=d))
    got = covariance_eigendecomposition_batched(sets)
    for X, (vecs, vals) in zip(sets, got):
        ref_vecs, ref_vals = sample_covariance_eigendecomposition(X)
        top = max(abs(ref_vals).max(), 1e-300)
        np.testing.assert_allclose(vals, ref_vals, rtol=0, atol=1e-12 * top)
        assert np.all(np.diff(vals) >= 0)
        C = np.cov(X, rowvar=False, ddof=1).reshape(d, d)
        np.testing.assert_allclose(vecs @ np.diag(vals) @ vecs.T, C, rtol=0, atol=1e-12 * top)
        np.testing.assert_allclose(vecs.T @ vecs, np.eye(d), rtol=0, atol=1e-13 * d)
        big = np.argmax(np.abs(vecs), axis=0)
        assert np.all(vecs[big, np.arange(d)] > 0)
        gaps = np.minimum(np.r_[np.inf, np.diff(ref_vals)], np.r_[np.diff(ref_vals), np.inf])
        sep = gaps > 1e-6 * top
        dots = np.abs(np.sum(vecs * ref_vecs, axis=0))
        np.testing.assert_allclose(dots[sep], 1.0, rtol=0, atol=1e-8)


def test_statuses_and_errors():
    import torch

    from art import _native as N
    from art._device import ptr
    from art.sampling import covariance_eigendecomposition_batched

    d = 3
    x = np.random.default_rng(1).normal(size=(10, d))
    x[7, 1] = np.nan
    ro = np.array([0, 1, 5, 10], dtype=np.int64)       # one row; fine; a NaN
    xt = torch.as_tensor(x.reshape(-1), device="cuda")
    rt = torch.as_tensor(ro, device="cuda")
    vals = torch.empty((3, d), dtype=torch.float64, device="cuda")
    vecs = torch.empty((3, d, d), dtype=torch.float64, device="cuda")
    st = torch.empty(3, dtype=torch.int32, device="cuda")
    lib = N.load_library()
    assert lib.art_covariance_eigh(ptr(xt), ptr(rt), 3, d, ptr(vals), ptr(vecs), ptr(st), None) == 0
    assert st.cpu().tolist() == [-1, 0, -2]
    v = vals.cpu().numpy()
    assert np.all(np.isnan(v[0])) and np.all(np.isfinite(v[1])) and np.all(np.isnan(v[2]))
    assert lib.art_covariance_eigh(ptr(xt), ptr(rt), 3, 65, ptr(vals), ptr(vecs), ptr(st), None) != 0
    with pytest.raises(ValueError):
        covariance_eigendecomposition_batched([x[:1]])
    with pytest.raises(ValueError):
        covariance_eigendecomposition_batched([x])
