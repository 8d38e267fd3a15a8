"""ctypes binding of the C ABI declared in ``include/art_b200.h``.

The library is loaded from the package tree (``lib/libart_b200.so``).  There
is no CPU fallback: every device entry point raises if the library or a CUDA
device is missing.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

from ._build import LIB_PATH

# ---- constants mirrored from include/art_b200.h ---------------------------
ART_OK = 0
ART_E_INVALID = -1
ART_E_WORKSPACE = -2
ART_E_LAUNCH = -3
ART_E_UNSUPPORTED = -4
ART_E_DEVICE = -5

FEATURES_AFFINE = 0
FEATURES_POLY1 = 1
FEATURES_POLY2 = 2
FEATURES_POLY1_NOBIAS = 3
FEATURES_POLY2_NOBIAS = 4

SOLVER_NORMAL = 0
SOLVER_AUTO = 1
SOLVER_QR = 2
SOLVER_SVD = 3
PRECISION_FP64 = 0
PRECISION_MIXED = 1

INFO_QR_FALLBACK = 1
INFO_RCOND_BELOW = 2
INFO_CHOLESKY_FAILED = 4
INFO_FP64_RESOLVE = 8
INFO_REFINE_CAP = 16
INFO_COND_FAILED = 32
INFO_REFINE_SHIFT = 8
INFO_SVD = 64
INFO_RANK_SHIFT = 16
MEDIAN_NN_MAX_SET = 4096
RIDGE_OPT_FP64_FACTOR = 1

MAX_FEATURES = 160
RIDGE_NOALLOC_MAX_COUNT = 65536
MAX_DIM = 64

HAR_BATCHED = 0
HAR_SCALAR = 1

STOP_REASONS = (
    "max_iters",
    "gradient_tolerance",
    "non_descent_direction",
    "line_search_failed",
    "max_line_search_failures",
    "alpha_min_reached",
)
SPLIT_FAILURES = (None, "cholesky_failure", "min_side_points", "nonfinite_split", "invalid_split")

P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32
F64 = C.c_double
U64 = C.c_uint64


class ArtSegments(C.Structure):
    _fields_ = [("count", I64), ("row_offsets", P), ("x_offsets", P), ("dims", P), ("features", P)]


class ArtRidgeProblem(C.Structure):
    _fields_ = [
        ("seg", ArtSegments), ("x", P), ("y", P), ("w", P), ("ridge", P),
        ("weight_floor", F64), ("solver", I32), ("precision", I32),
        ("auto_rcond_threshold", F64), ("max_features", I32), ("max_dim", I32),
        ("options", C.c_uint32), ("tensor_min_features", I32),
    ]


class ArtRidgeResult(C.Structure):
    _fields_ = [
        ("beta", P), ("beta_stride", I64), ("ridge_effective", P), ("cond_estimate", P),
        ("status", P), ("info", P),
    ]


class ArtSplitParams(C.Structure):
    _fields_ = [
        ("max_iters", I32), ("n_restarts", I32), ("grad_atol", F64), ("grad_rtol", F64),
        ("min_side_points", I32), ("min_side_fraction", F64), ("alpha0", F64), ("rho", F64),
        ("armijo_c", F64), ("max_backtracks", I32), ("adaptive_alpha", I32),
        ("alpha_min", F64), ("alpha_max", F64), ("alpha_grow", F64), ("alpha_recovery", F64),
        ("heavy_backtrack_threshold", I32), ("max_line_search_failures", I32),
        ("weight_floor", F64), ("hard_refit", I32), ("precision", I32),
        ("anneal_ratio", F64), ("seed", U64), ("group_restarts", I32), ("trial_steps", I32),
        ("ctas_per_sm", I32), ("tensor_gram", I32), ("restart_warps", I32),
    ]


class ArtSplitProblem(C.Structure):
    _fields_ = [
        ("seg", ArtSegments), ("x", P), ("y", P), ("temperature", P), ("ridge", P),
        ("parent_loss", P), ("min_side_fallback", P), ("theta0", P), ("theta_stride", I64),
        ("max_dim", I32), ("max_features", I32), ("node_keys", P), ("min_side_points", P),
    ]


class ArtSplitResult(C.Structure):
    _fields_ = [
        ("theta", P), ("theta_stride", I64), ("beta", P), ("beta_stride", I64), ("loss", P),
        ("child_loss", P), ("ridge_effective", P), ("n_right", P), ("n_iters", P),
        ("stop_reason", P), ("failure", P), ("flags", P), ("fallback_iteration", P),
        ("final_alpha", P), ("trace_loss", P), ("trace_step", P), ("trace_backtracks", P),
        ("trace_grad_norm", P),
    ]


class ArtPolytopes(C.Structure):
    _fields_ = [
        ("count", I64), ("dim", I32), ("lo", P), ("hi", P), ("row_offsets", P), ("A", P),
        ("b", P), ("max_rows", I32), ("reserved", I32), ("direction_maps", P),
    ]


class ArtChains(C.Structure):
    _fields_ = [
        ("count", I64), ("polytope", P), ("x", P), ("seeds", P), ("directions", P),
        ("uniforms", P), ("mode", I32), ("burn_in", I32), ("thinning", I32), ("n_rounds", I32),
        ("counter_base", U64), ("samples", P), ("status", P),
    ]


# Every entry point of include/art_b200.h with its ctypes signature.
SIGNATURES = {
    "art_ridge_workspace_size": (C.c_size_t, [I64, I32]),
    "art_ridge_batched": (C.c_int, [C.POINTER(ArtRidgeProblem), C.POINTER(ArtRidgeResult), P, C.c_size_t, P]),
    "art_ridge_noalloc_scratch_bytes": (C.c_size_t, []),
    "art_ridge_batched_noalloc": (C.c_int, [C.POINTER(ArtRidgeProblem), C.POINTER(ArtRidgeResult), P]),
    "art_ridge_gram": (C.c_int, [C.POINTER(ArtRidgeProblem), P, I64, P, P, C.c_size_t, P]),
    "art_split_workspace_size": (C.c_size_t, [I64, I32, I32, I32]),
    "art_split_level": (C.c_int, [C.POINTER(ArtSplitProblem), C.POINTER(ArtSplitParams),
                                  C.POINTER(ArtSplitResult), P, C.c_size_t, P]),
    "art_hit_and_run": (C.c_int, [C.POINTER(ArtPolytopes), C.POINTER(ArtChains), P]),
    "art_partition_rows": (C.c_int, [C.POINTER(ArtSegments), P, P, I64, P, P, P, P]),
    "art_segment_residuals": (C.c_int, [C.POINTER(ArtSegments), P, P, P, I64, P, P, P]),
    "art_tree_predict": (C.c_int, [I32, I64, P, P, I64, P, I64, P, I64, P, P, P, P]),
    "art_median_nn_distance": (C.c_int, [I64, P, P, P, P, P, I32, F64, P, P]),
    "art_covariance_eigh": (C.c_int, [P, P, I64, I32, P, P, P, P]),
    "art_last_error": (C.c_char_p, []),
    "art_abi_version": (C.c_int, []),
    "art_launch_count": (C.c_uint64, []),
    "art_profile_enable": (None, [C.c_int]),
    "art_profile_report": (C.c_int, [C.c_char_p, C.c_size_t]),
    "art_profile_reset": (None, []),
}

_lib = None
_lock = threading.Lock()


def library_path() -> Path:
    return LIB_PATH


def load_library(path: Path | None = None):
    """Load (once) and return the ctypes handle of ``libart_b200.so``."""

    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        lib_path = Path(path) if path is not None else LIB_PATH
        if not lib_path.exists():
            raise RuntimeError(
                f"{lib_path} is missing: build it with art._build.build() "
                "(nvcc, sm_100a). There is no CPU fallback."
            )
        lib = C.CDLL(str(lib_path))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        if lib.art_abi_version() != 1:
            raise RuntimeError("libart_b200.so ABI version mismatch")
        _lib = lib
        return lib


def last_error() -> str:
    lib = load_library()
    msg = lib.art_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != ART_OK:
        raise RuntimeError(f"{what} failed with code {rc}: {last_error()}")


def launch_count() -> int:
    return int(load_library().art_launch_count())


_profiling = False


def profile_enable(on: bool = True) -> None:
    global _profiling
    load_library().art_profile_enable(1 if on else 0)
    _profiling = bool(on)


def profiling() -> bool:
    """Whether the library's per-launch profiler was last switched on."""

    return _profiling


def profile_reset() -> None:
    load_library().art_profile_reset()


def profile_report() -> dict[str, tuple[int, float]]:
    """{kernel name: (launches, total ms)} for kernels launched while enabled."""

    buf = C.create_string_buffer(1 << 16)
    load_library().art_profile_report(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, n, ms = line.rsplit(" ", 2)
        out[name] = (int(n), float(ms))
    return out
