"""B200-native ART level-wise tree build (drop-in for the reference ``art`` package).

The numeric hot path -- weighted ridge fits, soft oblique split search and
hit-and-run sampling -- runs in hand-written sm_100a kernels reached through
the C ABI of ``include/art_b200.h``; PyTorch provides device memory and
streams.  Importing the package needs no GPU; calling a device entry point
does, and raises if no CUDA device or built library is present.
"""

from ._batched_optimizer import BatchedOptimizerWorkspace, optimize_batch
from .builder import LevelSplitDispatcher, RegressionTreeBuilder, TreeBuildResult
from .domain import BoxDomain, PolytopeRegion, split_region
from .metrics import (
    max_pointwise_relative_error,
    mean_squared_error,
    median_pointwise_relative_error,
    pointwise_relative_error,
    pointwise_relative_error_quantile,
    relative_l2_error,
    sum_squared_error,
)
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
    ridge_gram_batched,
    ridge_solve_diagnostics,
    scaled_ridge_from_gram,
    solve_weighted_ridge,
    solve_weighted_ridge_batched,
)
from .optimizers import AdaptiveAlpha, LineSearchResult, armijo_backtracking
from .presets import (
    B200_TREE_PRESET,
    BFS_GPU_TREE_PRESET,
    DEFAULT_TREE_PRESET,
    HingeAffinePreset,
    SamplingPreset,
    SoftObliquePreset,
    TemperaturePreset,
    TreePreset,
)
from .sampling import (
    BatchedHitAndRunSampler,
    HitAndRunSampler,
    NumbaBatchedHitAndRunSampler,
    ParallelNumbaBatchedHitAndRunSampler,
    Sampler,
    UniformBoxSampler,
    autocorrelation_by_lag,
    device_polytopes,
    find_feasible_point,
    floor_covariance_eigenvalues,
    hit_and_run_device,
    infer_box_bounds,
    covariance_eigendecomposition_batched,
    sample_covariance_eigendecomposition,
    sample_uniform_box,
)
from .splitters import (
    LevelResult,
    SoftObliqueSplitter,
    SplitNotFoundError,
    SplitResult,
    Splitter,
    project_unit_w,
    project_unit_w_gradient,
    split_level,
)
from .temperature import (
    DEFAULT_TEMPERATURE_GRID,
    TemperatureConfig,
    estimate_temperature,
    median_nearest_neighbor_distance,
    median_pairwise_distance,
    pairwise_distances,
    subsample_points,
    temperature_grid,
)
from .tree import LeafNode, RegressionTree, SplitNode

__version__ = "0.1.0"
