"""The C-ABI library loads (no GPU needed) and exports exactly what include/art_b200.h declares."""

import re
import subprocess

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "art_b200.h").read_text()
    return sorted(set(re.findall(r"ART_API\s+[\w\s\*]+?\b(art_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib):
    from art import _native

    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_native.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (art_\w+)", out))
    assert exported == set(names)


def test_abi_version_and_error_text(lib):
    assert lib.art_abi_version() == 1
    assert isinstance(lib.art_last_error(), bytes)


def test_host_validation_rejects_bad_arguments_without_launching(lib):
    import ctypes as C

    from art import _native as N

    before = lib.art_launch_count()
    assert lib.art_ridge_batched(None, None, None, 0, None) == N.ART_E_INVALID
    assert b"null" in lib.art_last_error()
    prob = N.ArtRidgeProblem()
    prob.seg.count = 3
    res = N.ArtRidgeResult()
    assert lib.art_ridge_batched(C.byref(prob), C.byref(res), None, 0, None) == N.ART_E_INVALID
    assert lib.art_hit_and_run(None, None, None) == N.ART_E_INVALID
    assert lib.art_launch_count() == before


def test_workspace_sizes_are_monotone(lib):
    a = lib.art_ridge_workspace_size(10, 9)
    b = lib.art_ridge_workspace_size(10000, 153)
    assert 0 < a < b
