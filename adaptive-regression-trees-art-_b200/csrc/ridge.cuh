// ridge.cuh -- definitions shared by the ridge kernels (plain FP64, mixed
// tensor-core, QR fallback) and the host entry point.
#pragma once
#include "common.cuh"
#include "bulk.cuh"
#include "linalg.cuh"

namespace art {

constexpr int kRidgeThreads = 256;
constexpr int kBuckets = 64;
// Work lists.  The plan kernels fill the first three; solve kernels append
// to the last two.
enum RidgeClass {
  CLS_SMALL = 0,    // FP64, 24 < (p+1) <= 48: 4x4 register tiles + row slices
  CLS_LARGE = 1,    // FP64, (p+1) > 48: 8x8 register tiles
  CLS_TENSOR = 2,   // mixed form, p > 32: tcgen05 split-product Gram
  CLS_WARP = 3,     // FP64, (p+1) <= 24: one warp per system
  CLS_QR = 4,       // auto solver fallback: Householder QR
  CLS_RESOLVE = 5,  // mixed form systems re-solved by the FP64 form
  kClasses = 6
};
constexpr int kPlanClasses = 4;
constexpr int kWarpMaxAug = 24;
constexpr int kSmallMaxAug = 48;
constexpr int kTensorMinP = 33;

struct RidgeArgs {
  int64_t K;
  const int64_t* row_offsets;
  const int64_t* x_offsets;
  const int32_t* dims;
  const int32_t* features;
  const double* x;
  const double* y;
  const double* w;
  const double* ridge;
  double weight_floor;
  int solver;
  int precision;
  double rcond_threshold;
  int pmax;
  int dmax;
  double* beta;
  int64_t beta_stride;
  double* ridge_eff;
  double* cond;
  int32_t* status;
  uint32_t* info;
  uint32_t options;
  int tensor_min_p;       // mixed form: smallest p on the tensor-core kernel
  float* gram_out;        // art_ridge_gram: packed tensor-core Grams
  int64_t gram_stride;
};

struct RidgeLists {
  int32_t* count;   // [kClasses]
  int32_t* cursor;  // [kClasses]
  int32_t* hist;    // [kPlanClasses][kBuckets]
  int32_t* start;   // [kPlanClasses][kBuckets]
  int32_t* err;     // [1] device-side error flag (bounded wait gave up)
  double* lambda;   // [K] effective ridge, kept for the QR fallback
  int32_t* list;    // [kClasses][K]
};

struct RidgeItem {
  int64_t r0, n, xoff;
  int d, kind, p;
  double ridge;
};

__device__ __forceinline__ RidgeItem load_item(const RidgeArgs& a, int k) {
  RidgeItem it;
  it.r0 = a.row_offsets[k];
  it.n = a.row_offsets[k + 1] - it.r0;
  it.xoff = a.x_offsets[k];
  it.d = a.dims[k];
  it.kind = a.features[k];
  it.p = feature_count(it.d, it.kind);
  it.ridge = a.ridge[k];
  return it;
}

__device__ __forceinline__ void push_list(const RidgeLists& L, int64_t K, int cls, int k) {
  int pos = atomicAdd(&L.count[cls], 1);
  L.list[(int64_t)cls * K + pos] = k;
}

__device__ __forceinline__ void write_failed(const RidgeArgs& a, int k, int p, int32_t status,
                                             double lam, uint32_t info) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  for (int i = threadIdx.x; i < p; i += blockDim.x) a.beta[(int64_t)k * a.beta_stride + i] = nan;
  if (threadIdx.x == 0) {
    a.status[k] = status;
    if (a.ridge_eff) a.ridge_eff[k] = lam;
    if (a.cond) a.cond[k] = nan;
    if (a.info) a.info[k] = info;
  }
}

// Finish a system whose augmented Gram [G h; h^T yWy] is in packed lower
// storage G (FP64, (p+1) rows) in shared memory: trace-scaled ridge, FP64
// Cholesky, solve, optional condition estimate, and the auto-solver policy
// of solve_weighted_ridge (models.py:268-371).  All threads call it.
// `vec` is shared scratch of >= 3*(p+1) doubles.  Returns true if the system
// was queued for the QR fallback.
template <int CT>
__device__ inline bool finish_fp64(const RidgeArgs& a, const RidgeLists& L, int k,
                                   const RidgeItem& it, double* G, int bad, double* vec,
                                   int* s_fail, double* s_scalar, uint32_t info0) {
  const int tid = threadIdx.x, p = it.p;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  // lambda = ridge * trace(G) / p   (scaled_ridge_from_gram, models.py:209-215)
  if (tid == 0) {
    double tr = 0.0;
    for (int i = 0; i < p; ++i) tr += G[pk(i, i)];
    double lam = it.ridge * tr / p;
    s_scalar[0] = lam;
    L.lambda[k] = lam;
  }
  __syncthreads();
  const double lam = s_scalar[0];
  if (bad) {
    write_failed(a, k, p, (bad & 2) ? -1 : -2, lam, info0);
    __syncthreads();
    return false;
  }
  if (a.solver == ART_SOLVER_QR || a.solver == ART_SOLVER_SVD) {  // explicit QR: no normal equations solve
    if (tid == 0) {
      if (a.ridge_eff) a.ridge_eff[k] = lam;
      if (a.cond) a.cond[k] = nan;
      if (a.info) a.info[k] = info0 | (a.solver == ART_SOLVER_SVD ? 0u : ART_INFO_QR_FALLBACK);
      a.status[k] = 0;
      push_list(L, a.K, CLS_QR, k);
    }
    __syncthreads();
    return true;
  }
  for (int i = tid; i < p; i += blockDim.x) G[pk(i, i)] += lam;
  __syncthreads();
  const bool want_cond = (a.cond != nullptr) || (a.solver == ART_SOLVER_AUTO);
  if (want_cond && tid < 32) {
    double an = warp_sym_norm1(G, p);
    if (tid == 0) s_scalar[1] = an;
  }
  __syncthreads();
  // wide systems: 32-column blocks; narrow ones keep the small-register form
  int fail;
  if constexpr (CT == 8) fail = chol_packed32<double>(G, p, s_fail);
  else fail = chol_packed<double, CT>(G, p, s_fail);
  if (fail) {
    if (a.solver == ART_SOLVER_AUTO) {
      if (tid == 0) {
        if (a.ridge_eff) a.ridge_eff[k] = lam;
        if (a.cond) a.cond[k] = __longlong_as_double(0x7ff0000000000000ll);  // inf
        if (a.info) a.info[k] = info0 | ART_INFO_QR_FALLBACK | ART_INFO_CHOLESKY_FAILED;
        a.status[k] = 0;
        push_list(L, a.K, CLS_QR, k);
      }
      __syncthreads();
      return true;
    }
    write_failed(a, k, p, fail, lam, info0);
    __syncthreads();
    return false;
  }
  double* z = vec;
  double* v = vec + (p + 1);
  double* sg = vec + 2 * (p + 1);
  if (tid < 32) {
    for (int i = tid; i < p; i += 32) z[i] = G[pk(p, i)];  // h
    __syncwarp();
    warp_forward<double, double>(G, z, p);
    warp_backward<double, double>(G, z, p);
    if (want_cond) {
      double est = warp_inv_norm1_estimate<double>(G, p, v, sg);
      if (tid == 0) {
        double an = s_scalar[1];
        double rcond = (est > 0.0 && isfinite(est) && an > 0.0) ? 1.0 / (an * est) : 0.0;
        s_scalar[2] = rcond;
      }
    }
  }
  __syncthreads();
  uint32_t info = info0;
  double cond = nan;
  if (want_cond) {
    double rcond = s_scalar[2];
    if (rcond > 0.0 && isfinite(rcond)) {
      cond = sqrt(1.0 / fmin(rcond, 1.0));
    } else {
      rcond = 0.0;
      cond = __longlong_as_double(0x7ff0000000000000ll);
      info |= ART_INFO_COND_FAILED;
    }
    if (a.solver == ART_SOLVER_AUTO && rcond < a.rcond_threshold) {
      if (tid == 0) {
        if (a.ridge_eff) a.ridge_eff[k] = lam;
        if (a.cond) a.cond[k] = cond;
        if (a.info) a.info[k] = info | ART_INFO_QR_FALLBACK | ART_INFO_RCOND_BELOW;
        a.status[k] = 0;
        push_list(L, a.K, CLS_QR, k);
      }
      __syncthreads();
      return true;
    }
  }
  int nonfinite = 0;
  for (int i = tid; i < p; i += blockDim.x) {
    double b = z[i];
    nonfinite |= !isfinite(b);
    a.beta[(int64_t)k * a.beta_stride + i] = b;
  }
  nonfinite = __syncthreads_or(nonfinite);
  if (tid == 0) {
    a.status[k] = nonfinite ? -3 : 0;
    if (a.ridge_eff) a.ridge_eff[k] = lam;
    if (a.cond) a.cond[k] = cond;
    if (a.info) a.info[k] = info;
  }
  __syncthreads();
  return false;
}

// Row of the lower-triangular tile grid holding linear tile index t.
__device__ __forceinline__ int tile_row(int t) {
  int I = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
  while (I * (I + 1) / 2 > t) --I;
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  return I;
}

// Host-side launch helpers (ridge.cu / ridge_tc.cu / ridge_warp.cu).
int launch_ridge_tensor(const RidgeArgs& a, const RidgeLists& L, cudaStream_t stream);
int launch_ridge_warp(const RidgeArgs& a, const RidgeLists& L, cudaStream_t stream);
int device_sm_count();

}  // namespace art
