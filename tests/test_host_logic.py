"""Host-side logic that needs no GPU: the ctypes mirror of the C ABI structs,
the autotuner's persistent table and candidate lists, graph shape classes, and
the slice boundaries of overlapped host staging."""

import ctypes as C
import json
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

STRUCTS = ["ArtSegments", "ArtRidgeProblem", "ArtRidgeResult", "ArtSplitParams", "ArtSplitProblem",
           "ArtSplitResult", "ArtPolytopes", "ArtChains"]


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """sizeof and field offsets of every ABI struct, from gcc on include/art_b200.h,
    equal the Python mirror's (a drifted mirror would pass garbage pointers)."""

    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import _native as N

    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "art_b200.h"', 'int main(void) {']
    for name in STRUCTS:
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in getattr(N, name)._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append('  return 0; }')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for name in STRUCTS:
        cls = getattr(N, name)
        assert int(out[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_autotune_table_persists_and_is_keyed_by_device(tmp_path, monkeypatch):
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import autotune

    path = tmp_path / "tune.json"
    monkeypatch.setenv("ART_AUTOTUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "device_key", lambda: "test-device|sm148|cc10.0")
    monkeypatch.setattr(autotune, "_LOADED", False)
    autotune.clear()
    try:
        assert autotune.cached_split_shape(16, 17, 16) == (0, 0, 0, 1)
        assert autotune.cached_ridge_choice() == (0, None)
        autotune._store(autotune._split_key(16, 17, 16), {"group_restarts": 8, "trial_steps": 2,
                                                                  "ctas_per_sm": 2})
        autotune._store(autotune._ridge_key(), {"tensor_min_features": 153, "fp64_factor": False})
        saved = json.loads(path.read_text())
        assert len(saved) == 2
        autotune.clear()
        monkeypatch.setattr(autotune, "_LOADED", False)
        assert autotune.cached_split_shape(16, 17, 16) == (8, 2, 2, 0)    # reloaded from the file
        assert autotune.cached_ridge_choice() == (153, False)
        monkeypatch.setattr(autotune, "device_key", lambda: "other-device|sm132|cc9.0")
        assert autotune.cached_split_shape(16, 17, 16) == (0, 0, 0, 1)    # another device: untuned
    finally:
        autotune.clear()


@pytest.mark.parametrize("R,backtracks", [(1, 25), (2, 25), (16, 25), (16, 3)])
def test_split_candidates_respect_thread_and_backtrack_limits(R, backtracks):
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art import autotune

    cands = autotune.split_candidates(R, backtracks, 16, 17)
    assert cands and len(set(cands)) == len(cands)
    for g, h, c, w in cands:
        if w:
            assert g == 0 and c == 0 and 1 <= h <= min(8, backtracks + 1)
            continue
        assert 1 <= g <= min(R, 16)
        assert 1 <= h <= min(32, 256 // g, backtracks + 1)
        assert c in (1, 2) and (c == 1 or g <= 8)
    assert {c for _, _, c, w in cands if not w} == {1, 2}
    assert any(w for *_, w in cands)
    # too wide for the warp form, or with the tensor-core Gram: CTA shapes only
    assert not any(w for *_, w in autotune.split_candidates(R, backtracks, 24, 25))
    assert not any(w for *_, w in autotune.split_candidates(R, backtracks, 16, 17, tensor_gram=True))


def test_graph_shape_classes_round_up_to_powers_of_two():
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art.graphs import _pow2

    assert [_pow2(v, 8) for v in (0, 1, 8, 9, 16, 17, 1000)] == [8, 8, 8, 16, 16, 32, 1024]
    assert _pow2(5000, 4096) == 8192 and _pow2(10, 4096) == 4096


def test_host_slice_bounds_cut_at_system_edges_with_equal_rows():
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art.models import host_slice_bounds

    rng = np.random.default_rng(3)
    n = rng.integers(1, 500, 1000)
    d = rng.integers(1, 17, 1000)
    ro = np.concatenate([[0], np.cumsum(n)])
    xo = np.concatenate([[0], np.cumsum(n * d)[:-1]])
    b = host_slice_bounds(ro, xo, d, 8)
    assert b[0] == 0 and b[-1] == 1000 and np.all(np.diff(b) > 0) and len(b) == 9
    rows = np.diff(ro[b])
    assert rows.max() < 1.2 * ro[-1] / 8                       # about equal shares of the rows
    assert host_slice_bounds(ro, xo, d, 1) is None               # one slice: no staging
    assert host_slice_bounds(ro[:2], xo[:1], d[:1], 8) is None   # one system
    gap = xo.copy(); gap[5:] += 3                                # x blocks not back to back
    assert host_slice_bounds(ro, gap, d, 8) is None
    assert host_slice_bounds(ro + 4, xo, d, 8) is None           # rows not from 0
    few = host_slice_bounds(ro[:4], xo[:3], d[:3], 8)            # more slices than systems
    assert few[0] == 0 and few[-1] == 3 and np.all(np.diff(few) > 0)


def test_temperature_method_names_are_checked_before_any_device_work():
    sys.path.insert(0, str(ROOT / "adaptive-regression-trees-art-_b200"))
    from art.temperature import median_nearest_neighbor_distance

    with pytest.raises(ValueError):
        median_nearest_neighbor_distance(np.zeros((4, 2)), method="ball_tree")
    assert median_nearest_neighbor_distance(np.array([[0.0, 0.0], [3.0, 4.0], [3.0, 4.5]]), method="bruteforce") == 0.5


def test_batched_optimizer_settings_validation_matches_reference_rules():
    """_cuda_batched_optimizer.py:59-85: model type, degree, line-search refits, parameter ranges."""
    import pytest

    from art import AffineRidgeModel, PolynomialRidgeModel, SoftObliqueSplitter
    from art._batched_optimizer import _batch_data, _dimensions, _node_ids, _validate_settings

    ok = SoftObliqueSplitter(AffineRidgeModel(ridge=1e-6), 0.1)
    _validate_settings(ok, 3, True)
    with pytest.raises(ValueError):
        _validate_settings(SoftObliqueSplitter(PolynomialRidgeModel(degree=3), 0.1), 3, True)
    with pytest.raises(ValueError):
        _validate_settings(SoftObliqueSplitter(AffineRidgeModel(), 0.1, rho=1.0), 3, True)
    with pytest.raises(ValueError):
        _validate_settings(ok, 3, "yes")
    with pytest.raises(ValueError):
        _dimensions(4, 0, 2)
    with pytest.raises(ValueError):
        _node_ids([1, 1], 4)
    assert list(_node_ids([2, 0], 4)) == [2, 0]
    with pytest.raises(ValueError):
        _batch_data(np.zeros((2, 3)), np.zeros(2), 1.0)
    with pytest.raises(ValueError):
        _batch_data(np.zeros((2, 3, 1)), np.zeros((2, 3)), 0.0)
