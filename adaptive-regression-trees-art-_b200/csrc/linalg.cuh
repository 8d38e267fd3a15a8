// linalg.cuh -- block-level dense kernels on packed lower-triangular storage
// in shared memory: blocked right-looking Cholesky, warp triangular solves,
// and a 1-norm condition estimate.  Used by every ridge/split solve.
//
// Packed index of (i, j), j <= i:  i*(i+1)/2 + j.
#pragma once
#include "common.cuh"

namespace art {

__host__ __device__ __forceinline__ int pk(int i, int j) { return i * (i + 1) / 2 + j; }

// 1 / v rounded to nearest: the same value as the division, with the
// reciprocal intrinsics
__device__ __forceinline__ float recip_rn(float v) { return __frcp_rn(v); }
__device__ __forceinline__ double recip_rn(double v) { return __drcp_rn(v); }

// Blocked right-looking Cholesky of the leading p x p block of packed A
// (in place, lower factor).  All threads of the block must call it.  Returns
// 0 or the 1-based index of the first pivot that was not positive (the
// LAPACK dpotrf info convention the reference's status codes use,
// art/_cuda_batched_cholesky.py:52-55).  `s_fail` is a shared int.
template <typename T, int CT = 8>
__device__ int chol_packed(T* A, int p, int* s_fail) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthreads = blockDim.x;
  if (tid == 0) *s_fail = 0;
  __syncthreads();
  for (int j0 = 0; j0 < p; j0 += 8) {
    const int jb = min(8, p - j0);
    // (1) diagonal block: warp 0, lane i holds row j0+i of the block.
    if (warp == 0) {
      T row[8];
#pragma unroll
      for (int c = 0; c < 8; ++c)
        row[c] = (lane < jb && c <= lane) ? A[pk(j0 + lane, j0 + c)] : T(0);
      int fail = 0;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < jb && !fail) {
          T dc = __shfl_sync(0xffffffffu, row[c], c);
          if (!(dc > T(0)) || !isfinite((double)dc)) {
            fail = j0 + c + 1;
          } else {
            T lcc = sqrt(dc);
            if (lane == c) row[c] = lcc;
            else if (lane > c && lane < jb) row[c] = row[c] / lcc;
#pragma unroll
            for (int k = c + 1; k < 8; ++k) {
              T lkc = __shfl_sync(0xffffffffu, row[c], k);
              if (k < jb && lane >= k && lane < jb) row[k] -= row[c] * lkc;
            }
          }
        }
      }
      if (!fail && lane < jb) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c <= lane) A[pk(j0 + lane, j0 + c)] = row[c];
      }
      if (lane == 0 && fail) *s_fail = fail;
    }
    __syncthreads();
    if (*s_fail) return *s_fail;
    const int j1 = j0 + jb;
    // (2) panel: rows i >= j1, L[i, j0:j1] = A[i, j0:j1] * L_JJ^{-T}
    for (int i = j1 + tid; i < p; i += nthreads) {
      T a[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) a[c] = (c < jb) ? A[pk(i, j0 + c)] : T(0);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < jb) {
          T s = a[c];
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (k < c) s -= a[k] * A[pk(j0 + c, j0 + k)];
          a[c] = s / A[pk(j0 + c, j0 + c)];
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < jb) A[pk(i, j0 + c)] = a[c];
    }
    __syncthreads();
    // (3) trailing update of the lower triangle of A[j1:p, j1:p] in CTxCT tiles
    const int m = p - j1;
    if (m > 0) {
      const int nbt = (m + CT - 1) / CT;
      const int ntiles = nbt * (nbt + 1) / 2;
      for (int t = tid; t < ntiles; t += nthreads) {
        int I = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (I * (I + 1) / 2 > t) --I;
        while ((I + 1) * (I + 2) / 2 <= t) ++I;
        const int J = t - I * (I + 1) / 2;
        const int rb = j1 + CT * I, cb = j1 + CT * J;
        T acc[CT][CT];
#pragma unroll
        for (int i = 0; i < CT; ++i)
#pragma unroll
          for (int j = 0; j < CT; ++j) acc[i][j] = T(0);
        for (int c = 0; c < jb; ++c) {
          T ai[CT], bj[CT];
#pragma unroll
          for (int i = 0; i < CT; ++i) ai[i] = (rb + i < p) ? A[pk(rb + i, j0 + c)] : T(0);
#pragma unroll
          for (int j = 0; j < CT; ++j) bj[j] = (cb + j < p) ? A[pk(cb + j, j0 + c)] : T(0);
#pragma unroll
          for (int i = 0; i < CT; ++i)
#pragma unroll
            for (int j = 0; j < CT; ++j) acc[i][j] = fma(ai[i], bj[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < CT; ++i)
#pragma unroll
          for (int j = 0; j < CT; ++j) {
            const int r = rb + i, c = cb + j;
            if (r < p && c <= r) A[pk(r, c)] -= acc[i][j];
          }
      }
    }
    __syncthreads();
  }
  return 0;
}

// The same factorisation with 32-column blocks: the diagonal block is
// factored by warp 0 in registers (lane i holds row i of the block), the
// panel below it by one thread per row, and the trailing matrix is updated
// in 8x8 register tiles with a 32-deep inner loop -- four times fewer block
// steps (and block barriers) than chol_packed for the same arithmetic.
template <typename T>
__device__ int chol_packed32(T* A, int p, int* s_fail) {
  constexpr int NB = 32, CT = 8;
  // single precision (the preconditioner of the mixed form): pivots from the
  // hardware reciprocal square root, columns scaled by it, the panel solve
  // multiplied by the stored reciprocals; double precision divides exactly
  constexpr bool kFast = sizeof(T) == 4;
  __shared__ T s_inv[NB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthreads = blockDim.x;
  if (tid == 0) *s_fail = 0;
  __syncthreads();
  for (int j0 = 0; j0 < p; j0 += NB) {
    const int jb = min(NB, p - j0);
    if (warp == 0) {
      T row[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) row[c] = (lane < jb && c <= lane) ? A[pk(j0 + lane, j0 + c)] : T(0);
      int fail = 0;
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < jb && !fail) {
          const T dc = __shfl_sync(0xffffffffu, row[c], c);
          if (!(dc > T(0) && dc < T(INFINITY))) {  // not positive, or not finite
            fail = j0 + c + 1;
          } else {
            // no per-lane masks: rows and columns past jb are zero and stay
            // zero, and entries above the diagonal (lane < k) are updated
            // but never stored or read
            if constexpr (kFast) {
              const T inv = rsqrtf(dc);
              row[c] = lane == c ? dc * inv : row[c] * inv;
              if (lane == c) s_inv[c] = inv;
            } else {
              const T lcc = sqrt(dc);
              row[c] = lane == c ? lcc : row[c] / lcc;
            }
#pragma unroll
            for (int k = c + 1; k < NB; ++k) {
              const T lkc = __shfl_sync(0xffffffffu, row[c], k);
              row[k] = fma(-row[c], lkc, row[k]);
            }
          }
        }
      }
      if (!fail && lane < jb) {
#pragma unroll
        for (int c = 0; c < NB; ++c)
          if (c <= lane) A[pk(j0 + lane, j0 + c)] = row[c];
      }
      if (lane == 0 && fail) *s_fail = fail;
    }
    __syncthreads();
    if (*s_fail) return *s_fail;
    const int j1 = j0 + jb;
    // panel: rows i >= j1, L[i, j0:j1] = A[i, j0:j1] L_JJ^{-T}
    for (int i = j1 + tid; i < p; i += nthreads) {
      T a[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) a[c] = (c < jb) ? A[pk(i, j0 + c)] : T(0);
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < jb) {
          T sacc = a[c];
          const T* lr = A + pk(j0 + c, j0);
#pragma unroll
          for (int k = 0; k < NB; ++k)
            if (k < c) sacc -= a[k] * lr[k];
          if constexpr (kFast) a[c] = sacc * s_inv[c];
          else a[c] = sacc / lr[c];
        }
      }
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < jb) A[pk(i, j0 + c)] = a[c];
    }
    __syncthreads();
    // trailing update of the lower triangle of A[j1:p, j1:p] in CTxCT tiles
    const int m = p - j1;
    if (m > 0) {
      const int nbt = (m + CT - 1) / CT;
      const int ntiles = nbt * (nbt + 1) / 2;
      for (int t = tid; t < ntiles; t += nthreads) {
        int I = (int)((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
        while (I * (I + 1) / 2 > t) --I;
        while ((I + 1) * (I + 2) / 2 <= t) ++I;
        const int J = t - I * (I + 1) / 2;
        const int rb = j1 + CT * I, cb = j1 + CT * J;
        const T* ra[CT];
        const T* rc[CT];
#pragma unroll
        for (int i = 0; i < CT; ++i) {
          ra[i] = A + pk(min(rb + i, p - 1), j0);
          rc[i] = A + pk(min(cb + i, p - 1), j0);
        }
        T acc[CT][CT];
#pragma unroll
        for (int i = 0; i < CT; ++i)
#pragma unroll
          for (int j = 0; j < CT; ++j) acc[i][j] = T(0);
        for (int c = 0; c < jb; ++c) {
          T ai[CT], bj[CT];
#pragma unroll
          for (int i = 0; i < CT; ++i) ai[i] = ra[i][c];
#pragma unroll
          for (int j = 0; j < CT; ++j) bj[j] = rc[j][c];
#pragma unroll
          for (int i = 0; i < CT; ++i)
#pragma unroll
            for (int j = 0; j < CT; ++j) acc[i][j] = fma(ai[i], bj[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < CT; ++i)
#pragma unroll
          for (int j = 0; j < CT; ++j) {
            const int r = rb + i, c = cb + j;
            if (r < p && c <= r) A[pk(r, c)] -= acc[i][j];
          }
      }
    }
    __syncthreads();
  }
  return 0;
}

// In-place inverse of the packed lower-triangular factor L (p x p, positive
// diagonal): on return A holds X = L^{-1}, also lower triangular.  All
// threads of the block call it; `Y` is scratch for (p - 32) x 32 values.
//  1. Every 32 x 32 diagonal block is inverted independently, one warp per
//     block: lane c builds column c of X_jj by forward substitution in
//     registers (row i of L_jj read by every lane: broadcast loads).
//  2. Block columns right to left: with X[j1:, j1:] already inverted,
//     X[j1:, j0:j1] = -(X[j1:, j1:] L[j1:, j0:j1]) X_jj, the panel product
//     staged in Y.  Each step reads only finished blocks of X and the still
//     original panel of L, so the update is in place.
template <typename T>
__device__ void tri_inv_packed32(T* A, int p, T* Y) {
  constexpr int NB = 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthreads = blockDim.x, nwarps = nthreads >> 5;
  const int nb = (p + NB - 1) / NB;
  for (int jb = warp; jb < nb; jb += nwarps) {
    const int j0 = jb * NB, bs = min(NB, p - j0);
    T x[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      T s = T(0);
      if (i < bs) {
        const T* row = A + pk(j0 + i, j0);
#pragma unroll
        for (int k = 0; k < NB; ++k)
          if (k < i) s = fma(row[k], x[k], s);
        const T inv_d = recip_rn(row[i]);
        x[i] = (i == lane) ? inv_d : (i > lane ? -s * inv_d : T(0));
      } else {
        x[i] = T(0);
      }
    }
    __syncwarp();
    if (lane < bs) {
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i >= lane && i < bs) A[pk(j0 + i, j0 + lane)] = x[i];
    }
  }
  __syncthreads();
  for (int jb = nb - 2; jb >= 0; --jb) {
    const int j0 = jb * NB, bs = NB, j1 = j0 + NB, m = p - j1;
    // Y[i][c] = sum_{k <= i} X[j1+i][j1+k] L[j1+k][j0+c], 8-column strips
    for (int t = tid; t < m * (NB / 8); t += nthreads) {
      const int i = t >> 2, c0 = (t & 3) * 8;
      const T* xr = A + pk(j1 + i, j1);
      T acc[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] = T(0);
      for (int k = 0; k <= i; ++k) {
        const T xv = xr[k];
        const T* lr = A + pk(j1 + k, j0 + c0);
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = fma(xv, lr[u], acc[u]);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) Y[i * NB + c0 + u] = acc[u];
    }
    __syncthreads();
    // X[j1+i][j0+c] = -sum_{c' >= c} Y[i][c'] X_jj[c'][c]
    for (int t = tid; t < m * bs; t += nthreads) {
      const int i = t / bs, c = t - i * bs;
      T sacc = T(0);
      for (int c2 = c; c2 < bs; ++c2) sacc = fma(Y[i * NB + c2], A[pk(j0 + c2, j0 + c)], sacc);
      A[pk(j1 + i, j0 + c)] = -sacc;
    }
    __syncthreads();
  }
}

// v_out = X^T (X v) for X = L^{-1} from tri_inv_packed32 (the preconditioner
// M^{-1} = L^{-T} L^{-1}); block-wide, `t` is scratch of length p.
template <typename T>
__device__ void apply_inv_factor(const T* X, int p, const double* v, double* t, double* out) {
  const int tid = threadIdx.x, nthreads = blockDim.x;
  for (int i = tid; i < p; i += nthreads) {
    const T* row = X + pk(i, 0);
    double s = 0.0;
    for (int k = 0; k <= i; ++k) s = fma((double)row[k], v[k], s);
    t[i] = s;
  }
  __syncthreads();
  for (int j = tid; j < p; j += nthreads) {
    double s = 0.0;
    for (int i = j; i < p; ++i) s = fma((double)X[pk(i, j)], t[i], s);
    out[j] = s;
  }
  __syncthreads();
}

// Solve L z = b in place (z initially b), one warp, L packed lower.
template <typename T, typename V>
__device__ void warp_forward(const T* L, V* z, int p) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < p; ++j) {
    if (lane == 0) z[j] = z[j] / (V)L[pk(j, j)];
    __syncwarp();
    const V zj = z[j];
    for (int i = j + 1 + lane; i < p; i += 32) z[i] -= (V)L[pk(i, j)] * zj;
    __syncwarp();
  }
}
// Solve L^T x = z in place, one warp.
template <typename T, typename V>
__device__ void warp_backward(const T* L, V* z, int p) {
  const int lane = threadIdx.x & 31;
  for (int j = p - 1; j >= 0; --j) {
    if (lane == 0) z[j] = z[j] / (V)L[pk(j, j)];
    __syncwarp();
    const V xj = z[j];
    const T* row = L + pk(j, 0);
    for (int i = lane; i < j; i += 32) z[i] -= (V)row[i] * xj;
    __syncwarp();
  }
}

// 1-norm of the symmetric matrix held in packed lower storage (one warp).
template <typename T>
__device__ double warp_sym_norm1(const T* A, int p) {
  const int lane = threadIdx.x & 31;
  double best = 0.0;
  for (int i = lane; i < p; i += 32) {
    double s = 0.0;
    for (int j = 0; j < p; ++j) s += fabs((double)(j <= i ? A[pk(i, j)] : A[pk(j, i)]));
    best = fmax(best, s);
  }
  return warp_max(best);
}

// Estimate of ||A^{-1}||_1 for A = L L^T from its Cholesky factor, by the
// iterative 1-norm estimator of Hager (1984) as refined by Higham (1988,
// "FORTRAN codes for estimating the one-norm of a real or complex matrix",
// Algorithm 4.1): the same method LAPACK's dpocon uses through dlacn2.
// One warp; `v`, `s` are shared scratch vectors of length p (double).
template <typename T>
__device__ double warp_inv_norm1_estimate(const T* L, int p, double* v, double* sg) {
  const int lane = threadIdx.x & 31;
  auto solve = [&](double* z) {
    warp_forward<T, double>(L, z, p);
    warp_backward<T, double>(L, z, p);
  };
  auto norm1 = [&](const double* z) {
    double s = 0.0;
    for (int i = lane; i < p; i += 32) s += fabs(z[i]);
    return warp_sum(s);
  };
  if (p == 1) return 1.0 / ((double)L[0] * (double)L[0]);
  for (int i = lane; i < p; i += 32) v[i] = 1.0 / p;
  __syncwarp();
  solve(v);
  double est = norm1(v);
  for (int i = lane; i < p; i += 32) sg[i] = v[i] >= 0.0 ? 1.0 : -1.0;
  __syncwarp();
  for (int i = lane; i < p; i += 32) v[i] = sg[i];
  __syncwarp();
  solve(v);  // z = A^{-T} xi (A symmetric)
  int jlast = -1;  // -1: x is the uniform vector e/p, else x = e_jlast
  for (int iter = 0; iter < 5; ++iter) {
    // j = argmax |z_i| (first occurrence)
    double bv = -1.0, zsum = 0.0;
    int bj = 0x7fffffff;
    for (int i = lane; i < p; i += 32) {
      double a = fabs(v[i]);
      zsum += v[i];
      if (a > bv || (a == bv && i < bj)) { bv = a; bj = i; }
    }
    zsum = warp_sum(zsum);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      int oj = __shfl_xor_sync(0xffffffffu, bj, o);
      if (ov > bv || (ov == bv && oj < bj)) { bv = ov; bj = oj; }
    }
    // Converged when ||z||_inf <= z^T x.
    const double ztx = (jlast < 0) ? zsum / p : v[jlast];
    if (bv <= ztx) break;
    jlast = bj;
    __syncwarp();
    for (int i = lane; i < p; i += 32) v[i] = (i == bj) ? 1.0 : 0.0;
    __syncwarp();
    solve(v);
    double est_new = norm1(v);
    int same = 1;
    for (int i = lane; i < p; i += 32) same &= ((v[i] >= 0.0 ? 1.0 : -1.0) == sg[i]);
    same = __all_sync(0xffffffffu, same);
    if (same || est_new <= est) {
      est = fmax(est, est_new);
      break;
    }
    est = est_new;
    __syncwarp();
    for (int i = lane; i < p; i += 32) {
      sg[i] = v[i] >= 0.0 ? 1.0 : -1.0;
      v[i] = sg[i];
    }
    __syncwarp();
    solve(v);
  }
  // Alternative estimate with x_i = (-1)^i (1 + i/(p-1)).
  __syncwarp();
  for (int i = lane; i < p; i += 32) v[i] = ((i & 1) ? -1.0 : 1.0) * (1.0 + (double)i / (p - 1));
  __syncwarp();
  solve(v);
  double alt = 2.0 * norm1(v) / (3.0 * p);
  __syncwarp();
  return fmax(est, alt);
}

}  // namespace art
