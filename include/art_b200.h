/*
 * art_b200.h -- C ABI of the B200-native ART level-wise tree build.
 *
 * Everything here is `extern "C"`, takes plain pointers, sizes and a
 * cudaStream_t, and is stream-ordered: no entry point synchronises the host
 * unless its comment says so.  Device pointers are C-contiguous; the caller
 * owns every buffer, including the workspace sized by the matching
 * *_workspace_size function.  The library never calls cudaMalloc/cudaFree.
 *
 * Return value of every entry point: ART_OK (0) or a negative ART_E_* code
 * for a host-detected configuration error (nothing was launched; the text is
 * available from art_last_error()).  Per-item numerical outcomes are reported
 * in per-item status arrays, with the meanings of the reference's batched GPU
 * form (art/_cuda_batched_cholesky.py:52-55):
 *      0  ok
 *     >0  Cholesky pivot index (1-based) that was not positive
 *     -1  bad gate / weight (negative or non-finite weight)
 *     -2  non-finite input data (x or y)
 *     -3  solve failed (non-finite coefficients)
 *     -4  item shape outside the compiled limits (d, p, feature kind)
 *     -5  a bounded device wait gave up (the item was not computed)
 * Non-fatal events are reported separately in an ART_INFO_* bitfield.
 *
 * Segmented layout: K items (ridge systems, tree nodes) are node-sorted runs
 * of rows.  Item k owns rows [row_offsets[k], row_offsets[k+1]) of y and w,
 * and the row-major (n_k x d_k) block of x that starts at element
 * x_offsets[k].  Items may differ in n_k, d_k and feature kind.
 *
 * A workspace belongs to one stream at a time: calls that share a workspace
 * must not overlap on the GPU (the reference states the same rule for its
 * BatchedCholeskyWorkspace, art/_cuda_batched_cholesky.py:57-61).
 */
#ifndef ART_B200_H
#define ART_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* art_stream_t; /* == cudaStream_t */

#if defined(__GNUC__)
#define ART_API __attribute__((visibility("default")))
#else
#define ART_API
#endif

#define ART_ABI_VERSION 1

/* ---- return codes ------------------------------------------------------ */
#define ART_OK 0
#define ART_E_INVALID (-1)    /* bad argument (null pointer, size, enum)      */
#define ART_E_WORKSPACE (-2)  /* workspace too small                          */
#define ART_E_LAUNCH (-3)     /* CUDA launch/config error                     */
#define ART_E_UNSUPPORTED (-4)/* shape outside the compiled limits            */
#define ART_E_DEVICE (-5)     /* no sm_100 device / wrong architecture        */

/* ---- feature kinds (models.py:200-206, 557-694) ------------------------ */
#define ART_FEATURES_AFFINE 0        /* [x_1..x_d, 1]  bias LAST (AffineRidgeModel) */
#define ART_FEATURES_POLY1 1         /* [1, x_1..x_d]  (PolynomialRidgeModel deg 1) */
#define ART_FEATURES_POLY2 2         /* [1, x_i, x_i x_j (i<=j)] sklearn order     */
#define ART_FEATURES_POLY1_NOBIAS 3  /* [x_1..x_d]                                 */
#define ART_FEATURES_POLY2_NOBIAS 4  /* [x_i, x_i x_j (i<=j)]                      */

/* ---- ridge solver policy (models.py:218-371) ---------------------------- */
#define ART_SOLVER_NORMAL 0  /* Cholesky; failure -> status = pivot index     */
#define ART_SOLVER_AUTO 1    /* Cholesky + rcond; rcond < threshold or failure
                                -> FP64 Householder QR on [sqrt(W)Phi; sqrt(l)I] */
#define ART_SOLVER_QR 2      /* FP64 Householder QR directly (solver="qr")    */
#define ART_SOLVER_SVD 3     /* FP64 Householder QR, then a one-sided Jacobi SVD
                                of R: the minimum-norm least-squares solution,
                                singular values <= eps * max dropped
                                (solver="svd", LAPACK gelsd in the reference,
                                models.py:374-448); cond = s_max / s_min     */

/* ---- precision forms ---------------------------------------------------- */
#define ART_PRECISION_FP64 0   /* plain form: FP64 Gram, FP64 Cholesky        */
#define ART_PRECISION_MIXED 1  /* tcgen05 TF32 hi/lo split-product Gram with
                                  FP32 accumulation, FP32 Cholesky, FP64
                                  iterative refinement on residuals recomputed
                                  from the data in FP64; systems that do not
                                  converge are re-solved by the FP64 form     */

/* ---- non-fatal info bits (per item) ------------------------------------ */
#define ART_INFO_QR_FALLBACK 1u        /* Householder QR produced the solution */
#define ART_INFO_RCOND_BELOW 2u        /* ...because rcond < threshold         */
#define ART_INFO_CHOLESKY_FAILED 4u    /* ...because Cholesky failed           */
#define ART_INFO_FP64_RESOLVE 8u       /* mixed form re-solved in FP64         */
#define ART_INFO_REFINE_CAP 16u        /* refinement hit its iteration cap     */
#define ART_INFO_COND_FAILED 32u       /* condition estimate failed            */
#define ART_INFO_SVD 64u               /* the Jacobi SVD produced the solution
                                          (solver="svd", or auto after a
                                          non-finite QR solution)             */
/* bits 16..23 (SVD path only): the numerical rank of the augmented design  */
#define ART_INFO_RANK_SHIFT 16
/* bits 8..15: FP64 refinement passes used by the mixed form (0 otherwise)  */
#define ART_INFO_REFINE_SHIFT 8

/* ---- limits ------------------------------------------------------------- */
#define ART_MAX_FEATURES 160   /* p = features per system (ridge, split fits) */
#define ART_MAX_DIM 64         /* d = input dimension (split search, sampling) */
/* ridge systems accept d up to ART_MAX_FEATURES, so an explicit design matrix
   can be passed with ART_FEATURES_POLY1_NOBIAS (features = columns).        */

/* ======================================================================== */
/*  Segments                                                                 */
/* ======================================================================== */
typedef struct ArtSegments {
  int64_t count;              /* K                                          */
  const int64_t* row_offsets; /* device [K+1], nondecreasing, [0] = 0 not required */
  const int64_t* x_offsets;   /* device [K]; element offset of item k in x  */
  const int32_t* dims;        /* device [K]; d_k in [1, ART_MAX_DIM]        */
  const int32_t* features;    /* device [K]; ART_FEATURES_*                 */
} ArtSegments;

/* ======================================================================== */
/*  Batched weighted ridge                                                   */
/*  Replaces BatchedCholeskyWorkspace.fit (art/_cuda_batched_cholesky.py:  */
/*  273-332) and, per system, solve_weighted_ridge (art/models.py:218-371): */
/*     G = Phi^T diag(max(w, floor)) Phi,  h = Phi^T (max(w,floor) y),      */
/*     lambda = ridge * trace(G) / p,  (G + lambda I) beta = h.              */
/* ======================================================================== */
typedef struct ArtRidgeProblem {
  ArtSegments seg;
  const double* x;        /* device */
  const double* y;        /* device, one per row */
  const double* w;        /* device, one per row; NULL means all ones      */
  const double* ridge;    /* device [K]: ridge before trace scaling         */
  double weight_floor;    /* models.py:245-247 (1e-12 for soft fits)        */
  int32_t solver;         /* ART_SOLVER_*                                   */
  int32_t precision;      /* ART_PRECISION_*                                */
  double auto_rcond_threshold; /* models.py:20 default 1e-10                */
  int32_t max_features;   /* host-known upper bound of p over the batch     */
  int32_t max_dim;        /* host-known upper bound of d (0: use max_features) */
  uint32_t options;       /* ART_RIDGE_OPT_* bits                           */
  int32_t tensor_min_features; /* mixed form: systems with p >= this go to the
                                  tensor-core kernel, smaller ones to the FP64
                                  kernels (0: 33; > 160: none)               */
} ArtRidgeProblem;

/* Mixed form: factor the tensor-core Gram in FP64 instead of FP32 (fewer
   systems fall back to the FP64 form on ill-conditioned data; one CTA per
   SM instead of two).                                                        */
#define ART_RIDGE_OPT_FP64_FACTOR 1u

typedef struct ArtRidgeResult {
  double* beta;            /* device [K * beta_stride]; NaN on failure     */
  int64_t beta_stride;     /* >= max_features                              */
  double* ridge_effective; /* device [K] (may be NULL)                     */
  double* cond_estimate;   /* device [K] sqrt(1/rcond) (auto) (may be NULL)*/
  int32_t* status;         /* device [K]                                   */
  uint32_t* info;          /* device [K] ART_INFO_* (may be NULL)          */
} ArtRidgeResult;

ART_API size_t art_ridge_workspace_size(int64_t count, int32_t max_features);
/* Weighted Grams only, by the mixed form's tensor-core path: for every system
 * with 33 <= p <= 160 and d <= ART_MAX_DIM, G' = sum_k q_k phi_k phi_k^T from
 * TF32 hi/lo split products accumulated in FP32, written as the packed lower
 * triangle (row i holds G'[i][0..i]) at gram + k * gram_stride (floats), with
 * status[k] = 0; other systems get status -4.  The GPU Gram / host solve
 * split of the reference's hybrid optimizer (art/_cuda_hybrid_gram.py:115-169)
 * and the accuracy probe of the mixed form.                                  */
ART_API int art_ridge_gram(const ArtRidgeProblem* problem, float* gram, int64_t gram_stride,
                           int32_t* status, void* workspace, size_t workspace_bytes,
                           art_stream_t stream);
ART_API int art_ridge_batched(const ArtRidgeProblem* problem, const ArtRidgeResult* result,
                      void* workspace, size_t workspace_bytes, art_stream_t stream);

/* art_ridge_batched without a caller workspace (no counterpart in the
 * reference, which solves on the host).  For callers that cannot allocate
 * device memory at solve time -- a host loop embedded in another runtime's
 * memory pool, or a C/FFI caller with no device allocator of its own -- the
 * call uses a fixed scratch array compiled into the library and makes no
 * allocation.  At most ART_RIDGE_NOALLOC_MAX_COUNT systems per call
 * (ART_E_UNSUPPORTED beyond); results equal art_ridge_batched's.  The scratch
 * is shared by every call on a device: calls that may overlap (different
 * streams, or host threads, on the same device) race and must be ordered by
 * the caller.  The first call on each device resolves the scratch address and
 * may load the module, so make it before any stream capture.  Every
 * zero-initialised part of the scratch is cleared on the stream by each call. */
#define ART_RIDGE_NOALLOC_MAX_COUNT 65536
ART_API size_t art_ridge_noalloc_scratch_bytes(void);
ART_API int art_ridge_batched_noalloc(const ArtRidgeProblem* problem, const ArtRidgeResult* result,
                                      art_stream_t stream);

/* ======================================================================== */
/*  Soft oblique split search, one launch per tree level                     */
/*  Replaces BatchedOptimizerWorkspace.optimize                              */
/*  (art/_cuda_batched_optimizer.py:527-607) and, per node,                  */
/*  SoftObliqueSplitter.split / _optimize_from_initialization               */
/*  (art/splitters.py:252-601).  The whole projected-gradient loop, Armijo   */
/*  backtracking (optimizers.py:72-121), AdaptiveAlpha (optimizers.py:20-69),*/
/*  stop rules, last-feasible tracking, restarts and the hard partition run */
/*  on the device; the host reads results once.                              */
/* ======================================================================== */
typedef struct ArtSplitParams {
  int32_t max_iters;
  int32_t n_restarts;           /* R >= 1                                  */
  double grad_atol, grad_rtol;
  int32_t min_side_points;
  double min_side_fraction;
  double alpha0, rho, armijo_c;
  int32_t max_backtracks;
  int32_t adaptive_alpha;       /* bool                                    */
  double alpha_min, alpha_max, alpha_grow, alpha_recovery;
  int32_t heavy_backtrack_threshold;
  int32_t max_line_search_failures;
  double weight_floor;          /* soft fits                               */
  int32_t hard_refit;           /* bool: fit hard children + hard loss      */
  int32_t precision;            /* ART_PRECISION_FP64, or _MIXED: sigmoid gates
                                   in single precision, sums/solves FP64
                                   (see tensor_gram)                         */
  double anneal_ratio;          /* T_k = T * anneal_ratio^(k/(max_iters-1)); 1 = off */
  uint64_t seed;                /* Philox key for device initialisation     */
  int32_t group_restarts;       /* restarts sharing one CTA's row passes
                                   (0: the largest that fits, <= 16)         */
  int32_t trial_steps;          /* Armijo step sizes evaluated per trial pass
                                   (0: min(4, 256 / group, backtracks + 1))  */
  int32_t ctas_per_sm;          /* 0 or 1: one CTA per SM with the deepest row
                                   ring; 2: two CTAs per SM, each with at most
                                   110 KB of shared memory and 128 registers a
                                   thread (falls back to 1 when the level's
                                   layout does not fit)                      */
  int32_t tensor_gram;          /* mixed form only: 1 = the soft-pass side Grams
                                   on the tensor cores (tcgen05 kind::tf32,
                                   TF32 hi/lo products of vech([phi;y][phi;y]^T)
                                   and the gate weights, FP32 accumulation over
                                   128 rows, FP64 across) when the augmented
                                   model has at most 21 features; 0 = FP64 sums */
  int32_t restart_warps;        /* 1 = one warp per (node, restart): each warp
                                   streams its node's rows in 32-row tiles and
                                   runs its restart's loop with no block
                                   barriers (d <= 23, p <= 23, at most 8 trial
                                   steps, not with tensor_gram; group_restarts
                                   and ctas_per_sm are then unused); 0 = the
                                   restarts of a group share one CTA's row
                                   passes                                   */
} ArtSplitParams;

typedef struct ArtSplitProblem {
  ArtSegments seg;            /* features must be AFFINE/POLY1/POLY2 kinds   */
  const double* x;
  const double* y;
  const double* temperature;  /* device [K]                                 */
  const double* ridge;        /* device [K] child model ridge              */
  const double* parent_loss;  /* device [K]                                 */
  const int8_t* min_side_fallback; /* device [K] bool                      */
  const double* theta0;       /* device [K][R][d+1] or NULL (device init)   */
  int64_t theta_stride;       /* >= ART_MAX_DIM + 1 elements per (k, r)     */
  int32_t max_dim;            /* host-known max d over the batch            */
  int32_t max_features;       /* host-known max p                           */
  const uint64_t* node_keys;  /* device [K] or NULL: device restart draws keyed
                                 by (seed, node_keys[k], r) instead of
                                 (seed, k, r), so a node's draws do not depend
                                 on its position in the batch               */
  const int32_t* min_side_points; /* device [K] or NULL: per-node minimum side
                                 count in place of params->min_side_points,
                                 so nodes with different limits share a call */
} ArtSplitProblem;

/* stop reasons (splitters.py:424-488) */
#define ART_STOP_MAX_ITERS 0
#define ART_STOP_GRADIENT_TOLERANCE 1
#define ART_STOP_NON_DESCENT 2
#define ART_STOP_LINE_SEARCH_FAILED 3
#define ART_STOP_MAX_LINE_SEARCH_FAILURES 4
#define ART_STOP_ALPHA_MIN_REACHED 5
/* failure reasons (SplitNotFoundError.reason) */
#define ART_SPLIT_OK 0
#define ART_SPLIT_CHOLESKY_FAILURE 1
#define ART_SPLIT_MIN_SIDE_POINTS 2
#define ART_SPLIT_NONFINITE 3
#define ART_SPLIT_INVALID 4

typedef struct ArtSplitResult {
  double* theta;          /* device [K][theta_stride]: best [w, z]          */
  int64_t theta_stride;
  double* beta;           /* device [K][2][beta_stride] hard child models  */
  int64_t beta_stride;
  double* loss;           /* device [K] hard loss (hard_refit) else NaN     */
  double* child_loss;     /* device [K][2] left/right hard MSE             */
  double* ridge_effective;/* device [K][2]                                   */
  int32_t* n_right;       /* device [K]                                     */
  int32_t* n_iters;       /* device [K] of the chosen restart               */
  int32_t* stop_reason;   /* device [K] ART_STOP_*                          */
  int32_t* failure;       /* device [K] ART_SPLIT_*                         */
  int32_t* flags;         /* device [K] bit0 converged, bit1 min-side fallback used */
  int32_t* fallback_iteration; /* device [K]                               */
  double* final_alpha;    /* device [K]                                     */
  /* optional per-(node, restart) traces, NULL to skip:                     */
  double* trace_loss;     /* [K][R][max_iters+1] soft loss history          */
  double* trace_step;     /* [K][R][max_iters]   accepted step sizes        */
  int32_t* trace_backtracks; /* [K][R][max_iters]                           */
  double* trace_grad_norm;   /* [K][R][max_iters+1]                        */
} ArtSplitResult;

ART_API size_t art_split_workspace_size(int64_t count, int32_t n_restarts, int32_t max_dim,
                                int32_t max_features);
ART_API int art_split_level(const ArtSplitProblem* problem, const ArtSplitParams* params,
                    const ArtSplitResult* result, void* workspace,
                    size_t workspace_bytes, art_stream_t stream);

/* ======================================================================== */
/*  Hit-and-run in node polytopes                                           */
/*  Replaces sample_precomputed_chains(_parallel) (art/_numba_sampling.py:  */
/*  45-167), BatchedHitAndRunSampler._advance_batch (art/sampling.py:       */
/*  886-962) and HitAndRunSampler.sample (art/sampling.py:445-495).         */
/*  Polytope j: lo_j <= x <= hi_j (box rows handled structurally) and       */
/*  A_j x <= b_j for rows [row_offsets[j], row_offsets[j+1]) of A/b.        */
/* ======================================================================== */
#define ART_HAR_BATCHED 0  /* numba form: unnormalised Gaussian directions,
                              incremental slack, exact-zero product tests   */
#define ART_HAR_SCALAR 1   /* HitAndRunSampler form: unit directions, slack
                              recomputed each step, |A u| > 1e-14 tests,
                              samples at steps burn_in + k*thinning         */

typedef struct ArtPolytopes {
  int64_t count;
  int32_t dim;                /* d, same for all polytopes of a call         */
  const double* lo;           /* device [count][d] or NULL (no box rows)     */
  const double* hi;           /* device [count][d] or NULL                   */
  const int64_t* row_offsets; /* device [count+1] oblique rows               */
  const double* A;            /* device [rows][d]                            */
  const double* b;            /* device [rows]                               */
  int32_t max_rows;           /* host-known max oblique rows per polytope    */
  int32_t reserved;
  const double* direction_maps; /* device [count][d][d] or NULL: device-drawn
                                 directions of polytope j's chains are
                                 u = M_j z (covariance-shaped sampling,
                                 sampling.py:86-127); injected draws are used
                                 as given                                    */
} ArtPolytopes;

typedef struct ArtChains {
  int64_t count;
  const int32_t* polytope;    /* device [count]                             */
  double* x;                  /* device [count][d] in: start, out: last state */
  const uint64_t* seeds;      /* device [count] Philox keys (NULL if injected) */
  const double* directions;   /* device [count][steps][d] injected draws or NULL */
  const double* uniforms;     /* device [count][steps] injected draws or NULL */
  int32_t mode;               /* ART_HAR_*                                   */
  int32_t burn_in, thinning, n_rounds; /* steps = burn_in + n_rounds*thinning */
  uint64_t counter_base;      /* Philox counter offset (advance between calls) */
  double* samples;            /* device [n_rounds][count][d]                 */
  int32_t* status;            /* device [count]: 0 ok, 1 empty chord, 2 bad start */
} ArtChains;

ART_API int art_hit_and_run(const ArtPolytopes* polytopes, const ArtChains* chains,
                    art_stream_t stream);

/* ======================================================================== */
/*  Partition and routing                                                    */
/* ======================================================================== */
/* Stable node-sorted partition of each item's rows by the sign of
 * w_k . x - z_k (>= 0 -> right), builder.py:487-500 / splitters.py:618.
 * The side is the sign of the exact value of w . x - z (a compensated dot
 * product, with exact expansion arithmetic where that cannot decide), so a
 * point lands on the side exact arithmetic gives; numpy's rounded score can
 * differ only where its rounding error exceeds |w . x - z|.  Writes, per item, the left
 * rows then the right rows as indices into the input rows (perm), and
 * n_right[k].  theta is [K][theta_stride] = [w, z]; items with split[k]==0
 * are copied unchanged (all left).                                           */
ART_API int art_partition_rows(const ArtSegments* seg, const double* x, const double* theta,
                       int64_t theta_stride, const int8_t* split, int64_t* perm,
                       int32_t* n_right, art_stream_t stream);

/* Batched tree routing + leaf prediction (tree.py:124-165).  Nodes are a
 * flat array: child[node][0/1] (left/right, -1 for a leaf), theta[node] =
 * [w, z], leaf coefficients coef[node][coef_stride] with feature kind
 * features[node].  Writes leaf[n] (node index) and pred[n].                  */
/* Per segment k: sse[k] = sum (y - phi(x) . beta_k)^2 and ssy[k] = sum y^2
 * over its rows (FP64, fixed summation order) -- the leaf fit error of
 * relative_l2_error (metrics.py) for every node of a level at once.       */
ART_API int art_segment_residuals(const ArtSegments* seg, const double* x, const double* y,
                                  const double* beta, int64_t beta_stride, double* sse,
                                  double* ssy, art_stream_t stream);

ART_API int art_tree_predict(int32_t dim, int64_t n_nodes, const int32_t* child,
                     const double* theta, int64_t theta_stride, const double* coef,
                     int64_t coef_stride, const int32_t* features, int64_t n_points,
                     const double* x, int32_t* leaf, double* pred, art_stream_t stream);

/* ======================================================================== */
/*  Temperature estimate                                                     */
/* ======================================================================== */
/* Median nearest-neighbour distance of K point sets, times c: the
 * "median_nn" mode of estimate_temperature (temperature.py:116-137, with
 * median_nearest_neighbor_distance 73-101).  The reference's kd-tree query
 * (k = 2) is replaced by an exact brute-force search in FP64.  Set k holds
 * rows sample_rows[sample_offsets[k] .. sample_offsets[k+1]) (row indices
 * into the row-major points at x + x_offsets[k], dims[k] columns each); the
 * caller draws the subsample (subsample_points, temperature.py:47-62).
 * temperature[k] = c * median over i of min over j != i of ||x_i - x_j||;
 * NaN for sets of fewer than two points.  max_set (the host-known largest
 * set) must not exceed ART_MEDIAN_NN_MAX_SET; it sizes the kernel's shared
 * arrays, and a set larger than max_set gets NaN (it is not processed).    */
#define ART_MEDIAN_NN_MAX_SET 4096
ART_API int art_median_nn_distance(int64_t count, const double* x, const int64_t* x_offsets,
                           const int32_t* dims, const int64_t* sample_offsets,
                           const int64_t* sample_rows, int32_t max_set, double c,
                           double* temperature, art_stream_t stream);

/* Sample covariance and its eigendecomposition for `count` point sets of
 * dimension dim <= 64 (the pilot-chain spectrum of the covariance-shaped
 * sampler: sample_covariance_eigendecomposition, sampling.py:86-106, called
 * per child at builder.py:1141-1200).  Set k holds rows
 * [row_offsets[k], row_offsets[k+1]) of samples (row-major, dim doubles a
 * row); C = (X - mean)^T (X - mean) / (n - 1).  Writes eigenvalues [count][dim]
 * in ascending order and eigenvectors [count][dim][dim] with eigenvector j in
 * column j (numpy.linalg.eigh's layout); each eigenvector's largest-magnitude
 * component is positive.  status[k]: 0 converged, 1 not converged in 40
 * Jacobi sweeps, -1 fewer than two rows, -2 a non-finite sample (then NaN
 * outputs).                                                                  */
ART_API int art_covariance_eigh(const double* samples, const int64_t* row_offsets, int64_t count,
                                int32_t dim, double* eigenvalues, double* eigenvectors,
                                int32_t* status, art_stream_t stream);

/* ======================================================================== */
/*  Misc                                                                     */
/* ======================================================================== */
ART_API const char* art_last_error(void);  /* thread-local text of the last error  */
ART_API int art_abi_version(void);
/* Number of distinct kernels this library has launched in the calling
 * process (diagnostic; counts launches issued through the entry points).     */
ART_API uint64_t art_launch_count(void);

/* Kernel timing (diagnostic).  While enabled, every kernel launched by an
 * entry point is bracketed by CUDA events on its stream.  art_profile_report
 * synchronises on those events and writes one line per kernel name,
 * "name launches total_ms\n", into buf (truncated to len); it returns the
 * number of kernel names.  art_profile_reset clears the accumulators.       */
ART_API void art_profile_enable(int on);
ART_API int art_profile_report(char* buf, size_t len);
ART_API void art_profile_reset(void);

#ifdef __cplusplus
}
#endif
#endif /* ART_B200_H */
