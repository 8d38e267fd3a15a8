// common.cuh -- device helpers shared by the ART sm_100a kernels.
//
// Nothing in here allocates.  Kernels report per-item outcomes through
// status arrays; host-side configuration errors are recorded with
// art::set_error() and returned as negative ART_E_* codes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/art_b200.h"

namespace art {

// ---------------------------------------------------------------- host side
void set_error(const char* fmt, ...);
void count_launch();
int check_launch(const char* what);
// Profiling brackets around one kernel launch (no-ops unless enabled).
void prof_begin(const char* name, cudaStream_t s);
void prof_end(cudaStream_t s);
int device_sm_count();
// CTAs of `kern` (with `threads` threads and `dyn_smem` bytes of dynamic
// shared memory) that one SM holds at once.  Prefers the full shared-memory
// carveout for the kernel, then takes the larger of the runtime's occupancy
// answer and the count implied by the kernel's registers, its shared memory
// and the SM's thread and block limits.  At least 1.
int resident_ctas(const void* kern, int threads, size_t dyn_smem);

constexpr int kWarp = 32;

// ---------------------------------------------------------------- reductions
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum over all threads; `scratch` holds >= blockDim.x/32 values.
// Every thread receives the total (fixed summation order: deterministic).
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  T t = T(0);
  const int nw = (blockDim.x + 31) >> 5;
  for (int i = 0; i < nw; ++i) t += scratch[i];
  return t;
}

// ---------------------------------------------------------------- features
// Number of model features p for input dimension d (models.py:154-168,
// polynomial_feature_count; affine adds one bias column).
__host__ __device__ inline int feature_count(int d, int kind) {
  switch (kind) {
    case ART_FEATURES_AFFINE:
    case ART_FEATURES_POLY1: return d + 1;
    case ART_FEATURES_POLY1_NOBIAS: return d;
    case ART_FEATURES_POLY2: return 1 + d + d * (d + 1) / 2;
    case ART_FEATURES_POLY2_NOBIAS: return d + d * (d + 1) / 2;
    default: return -1;
  }
}

// Feature f of kind `kind` is the product x[a]*x[b] where a, b are indices
// into x or -1 for the constant 1.  Orders follow sklearn PolynomialFeatures
// (combinations_with_replacement, i outer) and the affine bias-last layout
// (models.py:200-206; art/_cuda_features.py:13-29 pins the same order).
__host__ __device__ inline void feature_factors(int d, int kind, int f, int& a, int& b) {
  a = -1;
  b = -1;
  int bias_first = (kind == ART_FEATURES_POLY1 || kind == ART_FEATURES_POLY2);
  if (kind == ART_FEATURES_AFFINE) {
    if (f < d) a = f;
    return;
  }
  if (bias_first) {
    if (f == 0) return;
    f -= 1;
  }
  if (f < d) {
    a = f;
    return;
  }
  f -= d;  // index into the degree-2 block
  int i = 0;
  while (f >= d - i) {
    f -= d - i;
    ++i;
  }
  a = i;
  b = i + f;
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror & Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), written from the
// published round function: two 32x32->64 multiplies per round with the
// multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 /
// 0xBB67AE85.
struct Philox4 {
  uint32_t v[4];
};
__host__ __device__ inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                   uint32_t c3, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0;
    k1 += W1;
  }
  Philox4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

// Uniform double in (0, 1) from 64 random bits: 53-bit mantissa, offset by
// half an ulp so that 0 is never produced (Box-Muller takes its log).
__host__ __device__ inline double u01_open(uint32_t hi, uint32_t lo) {
  uint64_t v = (((uint64_t)hi << 32) | lo) >> 11;  // 53 bits
  return ((double)v + 0.5) * (1.0 / 9007199254740992.0);
}
// Uniform double in [0, 1).
__host__ __device__ inline double u01_closed_open(uint32_t hi, uint32_t lo) {
  uint64_t v = (((uint64_t)hi << 32) | lo) >> 11;
  return (double)v * (1.0 / 9007199254740992.0);
}

// Standard normal pair from one Philox block by the Box-Muller transform
// (Box & Muller 1958), evaluated with CUDA's log/sqrt/sincospi.
__device__ inline void normal_pair(const Philox4& r, double& z0, double& z1) {
  double u1 = u01_open(r.v[0], r.v[1]);
  double u2 = u01_closed_open(r.v[2], r.v[3]);
  double rad = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  z0 = rad * c;
  z1 = rad * s;
}

// The same transform in single precision for directions drawn on the device:
// a direction only needs i.i.d. Gaussian coordinates (the chord arithmetic
// that uses it stays FP64), and CUDA's logf/sqrtf/sincospif cost a fraction
// of the double-precision functions.  24-bit uniforms: u1 in (0, 1), so the
// radius is finite (at most ~5.9).
__device__ inline void normal_pair_f32(const Philox4& r, double& z0, double& z1) {
  const float u1 = ((float)(r.v[0] >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = (float)(r.v[2] >> 8) * (1.0f / 16777216.0f);
  const float rad = sqrtf(-2.0f * logf(u1));
  float sn, cs;
  sincospif(2.0f * u2, &sn, &cs);
  z0 = (double)(rad * cs);
  z1 = (double)(rad * sn);
}

// ---------------------------------------------------------------- misc
__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// Exact-sign helpers for routing: TwoProduct / TwoSum (Ogita, Rump & Oishi,
// "Accurate sum and dot product", SIAM J. Sci. Comput. 2005).
// Written with explicit round-to-nearest intrinsics so the compiler cannot
// contract them into FMAs, which would break the error-free transformations.
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = __dmul_rn(a, b);
  e = fma(a, b, -p);
}
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
// Compensated w.x - z (Dot2): about twice working precision, so the sign
// matches the exact sign except for scores within ~1e-30 relative of 0.
// `mag` receives sum |x_i w_i| + |z|, the scale of Dot2's error bound.
__device__ inline double dot2_score(const double* x, const double* w, int d, double z, double* mag = nullptr) {
  double s = 0.0, c = 0.0, m = 0.0;
  for (int i = 0; i < d; ++i) {
    double p, e, t, f;
    two_prod(x[i], w[i], p, e);
    two_sum(s, p, t, f);
    s = t;
    c = __dadd_rn(c, __dadd_rn(f, e));
    m = __dadd_rn(m, fabs(p));
  }
  double t, f;
  two_sum(s, -z, t, f);
  c = __dadd_rn(c, f);
  if (mag) *mag = __dadd_rn(m, fabs(z));
  return __dadd_rn(t, c);
}

// Exact sign of x.w - z for the rare scores Dot2 cannot resolve: every
// product is split exactly (p + e, TwoProduct) and the 2d + 1 terms are
// summed exactly into a nonoverlapping expansion (Shewchuk, "Adaptive
// precision floating-point arithmetic and fast robust geometric predicates",
// Discrete Comput. Geom. 1997: Grow-Expansion with zero elimination); the
// expansion's largest component carries the sign of the exact sum.  Exact
// for inputs whose products do not underflow (|x_i w_i| above ~1e-292).
static __device__ __noinline__ bool exact_score_nonnegative(const double* x, const double* w, int d, double z) {
  double h[2 * ART_MAX_DIM + 2];
  int m = 0;
  auto grow = [&](double b) {
    double q = b;
    int k = 0;
    for (int i = 0; i < m; ++i) {
      double sum, err;
      two_sum(q, h[i], sum, err);
      q = sum;
      if (err != 0.0) h[k++] = err;
    }
    if (q != 0.0) h[k++] = q;
    m = k;
  };
  for (int i = 0; i < d && i < ART_MAX_DIM; ++i) {
    double p, e;
    two_prod(x[i], w[i], p, e);
    grow(p);
    grow(e);
  }
  grow(-z);
  return m == 0 || h[m - 1] > 0.0;
}

// Side of a split for routing and partitions: (x.w - z) >= 0 evaluated
// exactly, i.e. the sign of the real number x.w - z (a point exactly on the
// plane goes right, as numpy's >= 0 sends an exact zero).  Dot2 decides
// whenever its result exceeds its error bound (Ogita, Rump & Oishi:
// |res - s| <= u|s| + gamma_{2n}^2 sum|p_i|, taken here with a factor 8 of
// slack); the expansion decides the rest.
__device__ inline bool right_side(const double* x, const double* w, int d, double z) {
  double mag;
  const double r = dot2_score(x, w, d, z, &mag);
  const double u = 1.1102230246251565e-16;  // 2^-53
  const double n = 2.0 * d + 2.0;
  const double bound = 8.0 * n * n * u * u * mag;
  if (fabs(r) > bound) return r >= 0.0;
  return exact_score_nonnegative(x, w, d, z);
}

}  // namespace art
