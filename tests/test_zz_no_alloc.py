"""art_ridge_batched_noalloc: the fixed-scratch ridge entry point.

Collected last on purpose: the fixed scratch is process-wide device state,
so the file must pass both alone and after every other GPU test has used the
library.  Two calls in a row on different batches must each equal the
workspace entry point bit for bit (the second call sees the scratch the first
one left behind).
"""

import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _batch(K, seed, solver, precision, n_max=600, device=None):
    import torch

    from art import _native as N
    from art import workloads
    from art.models import _PRECISION_CODES, _SOLVER_CODES

    wl = workloads.ridge_systems(K, seed=seed, n_min=1, n_max=n_max, device=device)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a, dt: (a if isinstance(a, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(a))).to(
        device=dev, dtype=dt).contiguous()
    keep = dict(x=t(wl.x, torch.float64), y=t(wl.y, torch.float64), w=t(wl.w, torch.float64),
                ro=t(wl.row_offsets, torch.int64), xo=t(wl.x_offsets, torch.int64),
                dims=t(wl.dims, torch.int32), feats=t(wl.kinds, torch.int32),
                ridge=t(wl.ridge, torch.float64))
    ptr = lambda a: C.c_void_p(a.data_ptr())
    seg = N.ArtSegments(K, ptr(keep["ro"]), ptr(keep["xo"]), ptr(keep["dims"]), ptr(keep["feats"]))
    prob = N.ArtRidgeProblem(seg, ptr(keep["x"]), ptr(keep["y"]), ptr(keep["w"]), ptr(keep["ridge"]), 1e-12,
                             _SOLVER_CODES[solver], _PRECISION_CODES[precision], 1e-10,
                             int(wl.max_features), int(wl.max_dim), 0, 0)
    return prob, keep, int(wl.max_features)


def _result(K, P):
    import torch

    from art import _native as N

    out = dict(beta=torch.full((K, P), float("nan"), dtype=torch.float64, device="cuda"),
               lam=torch.empty(K, dtype=torch.float64, device="cuda"),
               cond=torch.empty(K, dtype=torch.float64, device="cuda"),
               status=torch.empty(K, dtype=torch.int32, device="cuda"),
               info=torch.empty(K, dtype=torch.int32, device="cuda"))
    ptr = lambda a: C.c_void_p(a.data_ptr())
    res = N.ArtRidgeResult(ptr(out["beta"]), P, ptr(out["lam"]), ptr(out["cond"]), ptr(out["status"]),
                           ptr(out["info"]))
    return res, out


def _host(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def _solve_both(lib, K, seed, solver, precision, n_max=600, device=None):
    import torch

    from art import _native as N

    prob, keep, P = _batch(K, seed, solver, precision, n_max, device)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    res_a, out_a = _result(K, P)
    res_b, out_b = _result(K, P)
    ws = torch.empty(lib.art_ridge_workspace_size(K, P), dtype=torch.uint8, device="cuda")
    N.check(lib.art_ridge_batched(C.byref(prob), C.byref(res_a), C.c_void_p(ws.data_ptr()), ws.numel(), stream),
            "art_ridge_batched")
    N.check(lib.art_ridge_batched_noalloc(C.byref(prob), C.byref(res_b), stream), "art_ridge_batched_noalloc")
    torch.cuda.synchronize()
    del keep
    return _host(out_a), _host(out_b)


@pytest.mark.parametrize("solver,precision", [("normal", "fp64"), ("auto", "fp64"), ("normal", "mixed")])
def test_noalloc_equals_workspace_entry_on_two_calls_in_a_row(lib, solver, precision):
    for K, seed in ((300, 11), (77, 12)):
        a, b = _solve_both(lib, K, seed, solver, precision)
        for key in ("beta", "lam", "status", "info"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"{key} K={K}")
        assert (a["status"] == 0).mean() > 0.5


def test_noalloc_at_the_scratch_limit_equals_workspace_entry(lib):
    """Exactly ART_RIDGE_NOALLOC_MAX_COUNT small systems: the whole fixed
    scratch is in use, twice in a row."""
    from art import _native as N

    for seed in (21, 22):
        a, b = _solve_both(lib, N.RIDGE_NOALLOC_MAX_COUNT, seed, "auto", "fp64", n_max=24, device="cuda")
        for key in ("beta", "lam", "status", "info"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"{key} seed={seed}")


def test_noalloc_rejects_batches_beyond_the_fixed_scratch(lib):
    from art import _native as N

    assert lib.art_ridge_noalloc_scratch_bytes() >= lib.art_ridge_workspace_size(N.RIDGE_NOALLOC_MAX_COUNT, 160)
    prob, keep, P = _batch(4, 3, "normal", "fp64")
    prob.seg.count = N.RIDGE_NOALLOC_MAX_COUNT + 1   # rejected on the host before any launch
    res, _ = _result(4, P)
    n0 = lib.art_launch_count()
    assert lib.art_ridge_batched_noalloc(C.byref(prob), C.byref(res), None) == N.ART_E_UNSUPPORTED
    assert b"fixed scratch" in lib.art_last_error()
    assert lib.art_launch_count() == n0
