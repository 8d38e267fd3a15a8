// eig.cu -- sample covariance and its symmetric eigendecomposition for many
// point sets at once: the direction spectrum of the covariance-shaped
// hit-and-run sampler (sampling.py:86-106 sample_covariance_eigendecomposition,
// builder.py:1141-1200 the pilot chain per child), on the device.
//
// One CTA per point set (d <= 64):
//  1. mean and covariance C = (X - m)^T (X - m) / (n - 1) in FP64 shared
//     memory, each entry summed over the rows in row order;
//  2. cyclic two-sided Jacobi (Golub & Van Loan, Alg. 8.4.3 with the
//     symmetric Schur rotation of Alg. 8.4.1): every sweep is d - 1 rounds of
//     a round-robin tournament, each round rotating d / 2 disjoint (p, q)
//     pairs at once (A <- J^T A J as a column pass then a row pass, V <- V J),
//     until the off-diagonal mass is below (1e-15 ||C||_F)^2 or 40 sweeps;
//  3. eigenvalues in ascending order (numpy.linalg.eigh's order), each
//     eigenvector's largest-magnitude component made positive (the first one
//     on ties), so the result is deterministic; numpy's signs are LAPACK's.
#include <cmath>

#include "art_b200.h"
#include "common.cuh"

namespace art {
namespace {

constexpr int kEigThreads = 256;
constexpr int kEigMaxDim = 64;
constexpr int kEigMaxSweeps = 40;

__global__ void __launch_bounds__(kEigThreads) cov_eigh_kernel(const double* __restrict__ x,
                                                               const int64_t* __restrict__ row_offsets, int d,
                                                               double* __restrict__ evals,
                                                               double* __restrict__ evecs,
                                                               int32_t* __restrict__ status) {
  extern __shared__ __align__(16) double sm[];
  const int ds = d | 1;  // odd row stride
  double* A = sm;                    // [d][ds]
  double* V = A + d * ds;            // [d][ds]
  double* mean = V + d * ds;         // [d]
  double* rc = mean + kEigMaxDim;    // [32] cosines, [32] sines
  double* rs = rc + kEigMaxDim / 2;
  double* red = rs + kEigMaxDim / 2;  // [kEigThreads / 32]
  __shared__ int s_flag;
  const int k = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t r0 = row_offsets[k], n = row_offsets[k + 1] - r0;
  const double* X = x + r0 * d;
  if (n < 2) {
    if (tid == 0) status[k] = -1;
    for (int i = tid; i < d; i += kEigThreads) evals[(int64_t)k * d + i] = NAN;
    for (int i = tid; i < d * d; i += kEigThreads) evecs[(int64_t)k * d * d + i] = NAN;
    return;
  }
  // ---- mean and covariance
  if (tid == 0) s_flag = 0;
  __syncthreads();
  for (int j = tid; j < d; j += kEigThreads) {
    double s = 0.0;
    bool fin = true;
    for (int64_t r = 0; r < n; ++r) {
      const double v = X[r * d + j];
      fin = fin && isfinite(v);
      s += v;
    }
    mean[j] = s / (double)n;
    if (!fin) atomicExch(&s_flag, 1);
  }
  __syncthreads();
  if (s_flag) {
    if (tid == 0) status[k] = -2;
    for (int i = tid; i < d; i += kEigThreads) evals[(int64_t)k * d + i] = NAN;
    for (int i = tid; i < d * d; i += kEigThreads) evecs[(int64_t)k * d * d + i] = NAN;
    return;
  }
  for (int e = tid; e < d * d; e += kEigThreads) {
    const int i = e / d, j = e - (e / d) * d;
    if (j > i) continue;
    const double mi = mean[i], mj = mean[j];
    double s = 0.0;
    for (int64_t r = 0; r < n; ++r) s = fma(X[r * d + i] - mi, X[r * d + j] - mj, s);
    const double c = s / (double)(n - 1);
    A[i * ds + j] = c;
    A[j * ds + i] = c;
  }
  for (int e = tid; e < d * d; e += kEigThreads) {
    const int i = e / d, j = e - (e / d) * d;
    V[i * ds + j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  // ---- Frobenius norm (fixed order: per-thread strided sums, then warps, then warp 0)
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < kEigThreads / 32; ++w) t += red[w];
    return t;
  };
  double f = 0.0;
  for (int e = tid; e < d * d; e += kEigThreads) {
    const double v = A[(e / d) * ds + e % d];
    f += v * v;
  }
  const double fro2 = block_sum(f);
  const double tol2 = 1e-30 * fro2;
  const int m = (d + 1) & ~1;  // players, one dummy when d is odd
  int sweeps = 0;
  bool conv = fro2 == 0.0;
  for (; sweeps < kEigMaxSweeps && !conv; ++sweeps) {
    double off = 0.0;
    for (int e = tid; e < d * d; e += kEigThreads) {
      const int i = e / d, j = e - (e / d) * d;
      if (i != j) off += A[i * ds + j] * A[i * ds + j];
    }
    if (block_sum(off) <= tol2) { conv = true; break; }
    for (int round = 0; round < m - 1; ++round) {
      // pair slot t: players L[t], L[m-1-t] of the circle (0 fixed, the rest rotated)
      auto player = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + round) % (m - 1); };
      if (tid < m / 2) {
        int p = player(tid), q = player(m - 1 - tid);
        if (p > q) { const int t = p; p = q; q = t; }
        double c = 1.0, s = 0.0;
        if (q < d) {
          const double apq = A[p * ds + q];
          if (apq != 0.0) {
            const double tau = (A[q * ds + q] - A[p * ds + p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        rc[tid] = c;
        rs[tid] = s;
      }
      __syncthreads();
      // columns: A <- A J, V <- V J
      for (int e = tid; e < (m / 2) * d; e += kEigThreads) {
        const int t = e / d, i = e - (e / d) * d;
        int p = player(t), q = player(m - 1 - t);
        if (p > q) { const int u = p; p = q; q = u; }
        if (q >= d) continue;
        const double c = rc[t], s = rs[t];
        const double ap = A[i * ds + p], aq = A[i * ds + q];
        A[i * ds + p] = c * ap - s * aq;
        A[i * ds + q] = s * ap + c * aq;
        const double vp = V[i * ds + p], vq = V[i * ds + q];
        V[i * ds + p] = c * vp - s * vq;
        V[i * ds + q] = s * vp + c * vq;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int e = tid; e < (m / 2) * d; e += kEigThreads) {
        const int t = e / d, j = e - (e / d) * d;
        int p = player(t), q = player(m - 1 - t);
        if (p > q) { const int u = p; p = q; q = u; }
        if (q >= d) continue;
        const double c = rc[t], s = rs[t];
        const double ap = A[p * ds + j], aq = A[q * ds + j];
        A[p * ds + j] = c * ap - s * aq;
        A[q * ds + j] = s * ap + c * aq;
      }
      __syncthreads();
    }
  }
  // ---- ascending order (ties by index), sign convention, outputs
  for (int j = tid; j < d; j += kEigThreads) {
    const double lj = A[j * ds + j];
    int rank = 0;
    for (int i = 0; i < d; ++i) {
      const double li = A[i * ds + i];
      rank += (li < lj || (li == lj && i < j)) ? 1 : 0;
    }
    int arg = 0;
    double big = -1.0;
    for (int i = 0; i < d; ++i) {
      const double a = fabs(V[i * ds + j]);
      if (a > big) { big = a; arg = i; }
    }
    const double sg = V[arg * ds + j] < 0.0 ? -1.0 : 1.0;
    evals[(int64_t)k * d + rank] = lj;
    for (int i = 0; i < d; ++i) evecs[(int64_t)k * d * d + (int64_t)i * d + rank] = sg * V[i * ds + j];
  }
  if (tid == 0) status[k] = conv ? 0 : 1;
}

}  // namespace
}  // namespace art

using namespace art;

extern "C" int art_covariance_eigh(const double* samples, const int64_t* row_offsets, int64_t count, int32_t dim,
                                   double* eigenvalues, double* eigenvectors, int32_t* status,
                                   art_stream_t stream) {
  cudaGetLastError();
  if (count < 0) { set_error("art_covariance_eigh: negative count"); return ART_E_INVALID; }
  if (count == 0) return ART_OK;
  if (!samples || !row_offsets || !eigenvalues || !eigenvectors || !status) {
    set_error("art_covariance_eigh: null device pointer");
    return ART_E_INVALID;
  }
  if (dim < 1 || dim > kEigMaxDim) {
    set_error("art_covariance_eigh: dim in [1, %d] required", kEigMaxDim);
    return ART_E_UNSUPPORTED;
  }
  const int ds = dim | 1;
  const size_t smem = (size_t)(2 * dim * ds + kEigMaxDim + kEigMaxDim + kEigThreads / 32) * sizeof(double);
  if (cudaFuncSetAttribute(cov_eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("art_covariance_eigh: cannot reserve %zu bytes of shared memory", smem);
    return ART_E_UNSUPPORTED;
  }
  cudaStream_t s = (cudaStream_t)stream;
  prof_begin("cov_eigh", s);
  cov_eigh_kernel<<<(unsigned)count, kEigThreads, smem, s>>>(samples, row_offsets, dim, eigenvalues,
                                                               eigenvectors, status);
  prof_end(s);
  count_launch();
  return check_launch("art_covariance_eigh");
}
