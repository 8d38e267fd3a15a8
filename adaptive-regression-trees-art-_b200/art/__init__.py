"""B200-native ART level-wise tree build (drop-in for the reference ``art`` package).

The numeric hot path -- weighted ridge fits, soft oblique split search and
hit-and-run sampling -- runs in hand-written sm_100a kernels reached through
the C ABI of ``include/art_b200.h``; PyTorch provides device memory and
streams.  Importing the package needs no GPU; calling a device entry point
does, and raises if no CUDA device or built library is present.
"""

from .models import (
    AffineRidgeModel,
    BatchedRidgeResult,
    ConditionEstimator,
    DEFAULT_AUTO_RCOND_THRESHOLD,
    MODEL_CONDITION_WARNING_THRESHOLD,
    PolynomialRidgeModel,
    PreparedDesign,
    PreparedFeatureModel,
    RegressionModel,
    RidgeSolveResult,
    RidgeSolver,
    WeightedNormalEquations,
    WeightedRegressionModel,
    augment_features,
    model_effective_dimension,
    polynomial_feature_count,
    ridge_solve_diagnostics,
    scaled_ridge_from_gram,
    solve_weighted_ridge,
    solve_weighted_ridge_batched,
)

__version__ = "0.1.0"
