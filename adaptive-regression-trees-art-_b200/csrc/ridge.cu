// ridge.cu -- batched weighted ridge solves over node-sorted segments.
//
// One call solves K independent systems (n_k rows, d_k inputs, p_k
// features) following solve_weighted_ridge (art/models.py:218-371):
//   G = Phi^T diag(max(w, floor)) Phi,  h = Phi^T (max(w, floor) y),
//   lambda = ridge * trace(G) / p,  (G + lambda I) beta = h.
// Features are generated on chip from x and never stored in HBM (the
// reference's batched form materialises Phi and W*Phi,
// art/_cuda_batched_cholesky_kernels.cu:138-148).
//
// Launch sequence (all stream-ordered, no host sync):
//   plan_hist -> plan_scan -> plan_scatter : per-class work lists, largest
//       cost first (log2 buckets of n*(p+1)^2), built on the device;
//   [mixed] ridge_tc_kernel                : tcgen05 Gram + refinement;
//   ridge_warp_kernel                      : FP64, (p+1) <= 24, warp per system;
//   ridge_fp64_kernel<4>, <8>              : persistent FP64 work queues
//       (<4>: Gram on the FP64 tensor cores, mma.sync m8n8k4; <8>: 8x8
//       FP64 register tiles);
//   ridge_fp64_kernel<8> on the resolve list (mixed systems that did not
//       converge); ridge_qr_kernel on the auto-solver fallback list.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>

#include <atomic>

#include "ridge.cuh"

namespace art {

// ====================================================================== plan
__device__ __forceinline__ int plan_class(const RidgeArgs& a, int p) {
  // direct least-squares solvers never take the normal equations, so their
  // systems skip the tensor-core Gram (Gram-only calls keep it)
  const bool direct = a.solver == ART_SOLVER_QR || a.solver == ART_SOLVER_SVD;
  if (a.precision == ART_PRECISION_MIXED && p >= a.tensor_min_p && (a.gram_out || !direct)) return CLS_TENSOR;
  if (a.gram_out) return -1;  // Gram-only calls cover tensor-class systems only
  if (p + 1 <= kWarpMaxAug) return CLS_WARP;
  return (p + 1 <= kSmallMaxAug) ? CLS_SMALL : CLS_LARGE;
}

__device__ __forceinline__ int plan_bucket(int64_t n, int p) {
  double cost = (double)(n + 1) * (double)(p + 1) * (double)(p + 1);
  int e = ilogb(cost);
  return kBuckets - 1 - max(0, min(kBuckets - 1, e));  // bucket 0 = largest
}

// Validate each item, pick its class and cost bucket, count.
__global__ void ridge_plan_hist(RidgeArgs a, RidgeLists L) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.K) return;
  const int d = a.dims[k], kind = a.features[k];
  const int p = feature_count(d, kind);
  const int64_t n = a.row_offsets[k + 1] - a.row_offsets[k];
  if (d < 1 || d > a.dmax || p < 1 || p > a.pmax || n < 0) {
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    a.status[k] = -4;
    if (a.ridge_eff) a.ridge_eff[k] = nan;
    if (a.cond) a.cond[k] = nan;
    if (a.info) a.info[k] = 0u;
    for (int i = 0; i < a.pmax; ++i) a.beta[k * a.beta_stride + i] = nan;
    return;
  }
  const int c = plan_class(a, p);
  if (c < 0) {
    a.status[k] = -4;
    return;
  }
  atomicAdd(&L.hist[c * kBuckets + plan_bucket(n, p)], 1);
}

__global__ void ridge_plan_scan(RidgeLists L) {
  // one block of kPlanClasses warps; warp c scans class c's buckets
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c >= kPlanClasses) return;
  int carry = 0;
  for (int base = 0; base < kBuckets; base += 32) {
    int v = L.hist[c * kBuckets + base + lane];
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    L.start[c * kBuckets + base + lane] = carry + incl - v;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) L.count[c] = carry;
}

__global__ void ridge_plan_scatter(RidgeArgs a, RidgeLists L) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.K) return;
  const int d = a.dims[k], kind = a.features[k];
  const int p = feature_count(d, kind);
  const int64_t n = a.row_offsets[k + 1] - a.row_offsets[k];
  if (d < 1 || d > a.dmax || p < 1 || p > a.pmax || n < 0) return;
  const int c = plan_class(a, p), b = plan_bucket(n, p);
  if (c < 0) return;
  const int slot = atomicSub(&L.hist[c * kBuckets + b], 1) - 1;
  L.list[(int64_t)c * a.K + L.start[c * kBuckets + b] + slot] = (int32_t)k;
}

// ============================================================ FP64 kernel
// Shared-memory layout, identical on host and device.
struct Fp64Layout {
  int ldp;        // max padded augmented width
  int chunk;
  size_t off_x[2], off_y[2], off_w[2], off_bar, off_phi, off_q, off_gram, off_fa, off_fb,
      off_vec, total;
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// Position of feature blk*TS + j in a row of the sqrt(q)*phi tile of the
// 8x8 register-tile form, and its row stride: within a block the entries
// rotate by the block index, which spreads a warp's loads over the banks.
__host__ __device__ inline int phi_pos(int ts, int blk, int j) { return blk * ts + ((j + blk) & (ts - 1)); }
__host__ __device__ inline int phi_stride(int ts, int nb) { return nb * ts; }

// Row stride of the phi tile in the 4-feature-block kernel, which forms the
// Gram with FP64 tensor-core MMAs (m8n8k4): 8-feature blocks, stride = 8
// (mod 16) doubles so that a fragment load (4 rows x 8 features) touches
// every bank pair exactly twice.
__host__ __device__ inline int dmma_stride(int pa) {
  const int nb8 = (pa + 7) / 8;
  return 8 * nb8 + ((nb8 & 1) ? 0 : 8);
}

// D (8x8, two doubles per lane) += A (8x4) * B (4x8) in FP64 on the tensor
// cores.  Lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__host__ __device__ inline Fp64Layout fp64_layout(int pmax, int dmax, int ts, int chunk) {
  Fp64Layout L;
  const int pa = pmax + 1;
  // features incl. padding: 8-feature blocks in the tensor-core form (ts = 4)
  L.ldp = ts == 4 ? ((pa + 7) / 8) * 8 : ((pa + ts - 1) / ts) * ts;
  L.chunk = chunk;
  size_t o = 0;
  for (int s = 0; s < 2; ++s) {
    L.off_x[s] = o; o = align16(o + (size_t)chunk * dmax * 8 + 16);
    L.off_y[s] = o; o = align16(o + (size_t)chunk * 8 + 16);
    L.off_w[s] = o; o = align16(o + (size_t)chunk * 8 + 16);
  }
  L.off_bar = o; o = align16(o + 2 * 8);
  L.off_phi = o;
  o = align16(o + (size_t)chunk * (ts == 4 ? dmma_stride(pa) : phi_stride(ts, L.ldp / ts)) * 8);
  L.off_q = o; o = align16(o + (size_t)chunk * 8);
  L.off_gram = o; o = align16(o + (size_t)pa * (pa + 1) / 2 * 8);
  L.off_fa = o; o = align16(o + (size_t)L.ldp * 2);
  L.off_fb = o; o = align16(o + (size_t)L.ldp * 2);
  L.off_vec = o; o = align16(o + (size_t)3 * (pa + 1) * 8);
  L.total = o;
  return L;
}

// Issue the bulk copies of chunk c (x rows, y, w) into stage st.
__device__ __forceinline__ void issue_chunk(const RidgeArgs& a, const RidgeItem& it, int chunk,
                                            int64_t c, unsigned char* smem, const Fp64Layout& lay,
                                            int st, uint64_t* bar) {
  const int64_t rr = c * chunk;
  const int rows = (int)min((int64_t)chunk, it.n - rr);
  Granules gx = granules(a.x + it.xoff + rr * it.d, (uint64_t)rows * it.d * 8);
  Granules gy = granules(a.y + it.r0 + rr, (uint64_t)rows * 8);
  Granules gw = a.w ? granules(a.w + it.r0 + rr, (uint64_t)rows * 8) : Granules{nullptr, 0, 0};
  mbar_arrive_expect_tx(bar, gx.bytes + gy.bytes + gw.bytes);
  bulk_g2s(smem + lay.off_x[st], gx.base, gx.bytes, bar);
  bulk_g2s(smem + lay.off_y[st], gy.base, gy.bytes, bar);
  if (a.w) bulk_g2s(smem + lay.off_w[st], gw.base, gw.bytes, bar);
}

// TS = 4 (tensor-core Gram, 80 registers) is held to three CTAs per SM.
template <int TS, int CHUNK>
__global__ void __launch_bounds__(kRidgeThreads, TS == 4 ? 3 : 1) ridge_fp64_kernel(RidgeArgs a, RidgeLists L,
                                                                   int cls, int pcap) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item, s_fail;
  __shared__ double s_scalar[4];
  const Fp64Layout lay = fp64_layout(pcap, a.dmax, TS, CHUNK);
  uint64_t* bars = (uint64_t*)(smem + lay.off_bar);
  double* phi = (double*)(smem + lay.off_phi);
  double* q = (double*)(smem + lay.off_q);
  double* G = (double*)(smem + lay.off_gram);
  int16_t* fa = (int16_t*)(smem + lay.off_fa);
  int16_t* fb = (int16_t*)(smem + lay.off_fb);
  double* vec = (double*)(smem + lay.off_vec);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0;  // completed phases per stage (uniform)
  const int count = L.count[cls];
  for (;;) {
    if (tid == 0) s_item = atomicAdd(&L.cursor[cls], 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= count) break;
    const int k = L.list[(int64_t)cls * a.K + item];
    const RidgeItem it = load_item(a, k);
    const int p = it.p, pa = p + 1, d = it.d;
    // TS = 4: FP64 tensor-core tiles of 8 features; TS = 8: 8x8 register tiles
    constexpr bool kDmma = TS == 4;
    const int nb = kDmma ? (pa + 7) / 8 : (pa + TS - 1) / TS;
    const int ldpi = kDmma ? 8 * nb : nb * TS;            // features incl. padding
    const int lds = kDmma ? dmma_stride(pa) : phi_stride(TS, nb);  // phi row stride
    const int T = nb * (nb + 1) / 2;
    const int S = kDmma ? 1 : max(1, kRidgeThreads / T);
    for (int f = tid; f < ldpi; f += kRidgeThreads) {
      int fa_, fb_;
      if (f < p) feature_factors(d, it.kind, f, fa_, fb_);
      else if (f == p) { fa_ = -2; fb_ = -1; }
      else { fa_ = -3; fb_ = -1; }
      fa[f] = (int16_t)fa_;
      fb[f] = (int16_t)fb_;
    }
    const bool mine = tid < T * S;
    const int tile = tid % T, slice = tid / T;
    const int I = tile_row(tile), J = tile - I * (I + 1) / 2;
    double acc[TS][TS];
#pragma unroll
    for (int i = 0; i < TS; ++i)
#pragma unroll
      for (int j = 0; j < TS; ++j) acc[i][j] = 0.0;
    // tensor-core form: warp w owns 8x8 tiles w, w + 8, w + 16 (T <= 21)
    const int wid = tid >> 5, wl = tid & 31;
    double dacc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    int tI[3], tJ[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int t2 = wid + 8 * m;
      tI[m] = t2 < T ? tile_row(t2) : 0;
      tJ[m] = t2 < T ? t2 - tI[m] * (tI[m] + 1) / 2 : 0;
    }
    int bad = 0;
    const int64_t nchunks = (it.n + CHUNK - 1) / CHUNK;
    if (tid == 0) {
      for (int64_t c = 0; c < min((int64_t)2, nchunks); ++c)
        issue_chunk(a, it, CHUNK, c, smem, lay, (int)c, &bars[c]);
    }
    __syncthreads();  // fa/fb visible
    bool timed_out = false;
    int64_t timed_c = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
      const int st = (int)(c & 1);
      const uint32_t par = st ? (uses1 & 1) : (uses0 & 1);
      const bool ok = mbar_wait(&bars[st], par);
      if (!__syncthreads_and(ok)) { timed_out = true; timed_c = c; break; }
      if (st) ++uses1; else ++uses0;
      const int rows = (int)min((int64_t)CHUNK, it.n - c * CHUNK);
      const double* xs =
          (const double*)(smem + lay.off_x[st] +
                          (((uintptr_t)(a.x + it.xoff + c * CHUNK * d)) & 15));
      const double* ys =
          (const double*)(smem + lay.off_y[st] + (((uintptr_t)(a.y + it.r0 + c * CHUNK)) & 15));
      const double* ws =
          a.w ? (const double*)(smem + lay.off_w[st] +
                                (((uintptr_t)(a.w + it.r0 + c * CHUNK)) & 15))
              : nullptr;
      for (int e = tid; e < rows * d; e += kRidgeThreads) bad |= isfinite(xs[e]) ? 0 : 1;
      for (int r = tid; r < rows; r += kRidgeThreads) {
        bad |= isfinite(ys[r]) ? 0 : 1;
        double wv = ws ? ws[r] : 1.0;
        if (!(wv >= 0.0) || !isfinite(wv)) bad |= 2;
        q[r] = sqrt(fmax(wv, a.weight_floor));
      }
      __syncthreads();
      // phi[r][phi_pos(blk, j)] = sqrt(q_r) * feature(blk*TS + j): the
      // rotation and shift spread the tiles' loads over distinct banks.
      const int warp = tid >> 5, lane = tid & 31;
      // the tensor-core form reads rows in groups of 4: pad with zero rows
      const int rows_pad = kDmma ? (rows + 3) & ~3 : rows;
      for (int r = warp; r < rows_pad; r += kRidgeThreads / 32) {
        const bool live = r < rows;
        const double* xr = xs + (int64_t)(live ? r : 0) * d;
        const double sq = live ? q[r] : 0.0;
        for (int f = lane; f < ldpi; f += 32) {
          const int ia = fa[f], ib = fb[f];
          double v;
          if (ia == -3 || !live) v = 0.0;
          else if (ia == -2) v = sq * ys[r];
          else v = sq * ((ia < 0 ? 1.0 : xr[ia]) * (ib < 0 ? 1.0 : xr[ib]));
          if constexpr (kDmma) {
            phi[r * lds + f] = v;
          } else {
            const int blk = f / TS, j = f - blk * TS;
            phi[r * lds + phi_pos(TS, blk, j)] = v;
          }
        }
      }
      __syncthreads();
      if (tid == 0 && c + 2 < nchunks) issue_chunk(a, it, CHUNK, c + 2, smem, lay, st, &bars[st]);
      if constexpr (kDmma) {
        const int off = (wl & 3) * lds + (wl >> 2);
        for (int k0 = 0; k0 < rows_pad; k0 += 4) {
          const double* pr = phi + k0 * lds + off;
#pragma unroll
          for (int m = 0; m < 3; ++m)
            if (wid + 8 * m < T) dmma_884(dacc[m], pr[8 * tI[m]], pr[8 * tJ[m]]);
        }
      } else if (mine) {
        for (int r = slice; r < rows; r += S) {
          const double* pr = phi + r * lds;
          double av[TS], bv[TS];
#pragma unroll
          for (int i = 0; i < TS; ++i) av[i] = pr[phi_pos(TS, I, i)];
#pragma unroll
          for (int j = 0; j < TS; ++j) bv[j] = pr[phi_pos(TS, J, j)];
#pragma unroll
          for (int i = 0; i < TS; ++i)
#pragma unroll
            for (int j = 0; j < TS; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
      }
      __syncthreads();
    }
    if (timed_out) {
      if (tid == 0) {
        atomicExch(L.err, 1);
        a.status[k] = -5;
        // bounded waits for this CTA's own copies still in flight
        for (int64_t c2 = timed_c; c2 < min(timed_c + 2, nchunks); ++c2) {
          const int s2 = (int)(c2 & 1);
          mbar_wait(&bars[s2], s2 ? (uses1 & 1) : (uses0 & 1));
          if (s2) ++uses1; else ++uses0;
        }
      }
      return;  // barrier phases are no longer consistent: stop this CTA
    }
    {
      const int bw = __syncthreads_or(bad & 2), bx = __syncthreads_or(bad & 1);
      bad = (bw ? 2 : 0) | (bx ? 1 : 0);
    }
    if constexpr (kDmma) {  // each lower entry belongs to one warp's tile
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        if (wid + 8 * m >= T) continue;
        const int r = 8 * tI[m] + (wl >> 2);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int cc = 8 * tJ[m] + 2 * (wl & 3) + e;
          if (r < pa && cc <= r) G[pk(r, cc)] = dacc[m][e];
        }
      }
      __syncthreads();
    }
    // deterministic slice reduction into the packed augmented Gram
    for (int s = 0; s < (kDmma ? 0 : S); ++s) {
      if (mine && slice == s) {
#pragma unroll
        for (int i = 0; i < TS; ++i)
#pragma unroll
          for (int j = 0; j < TS; ++j) {
            const int r = I * TS + i, cc = J * TS + j;
            if (r < pa && cc <= r) {
              double* g = &G[pk(r, cc)];
              *g = (s == 0) ? acc[i][j] : *g + acc[i][j];
            }
          }
      }
      __syncthreads();
    }
    finish_fp64<TS>(a, L, k, it, G, bad, vec, &s_fail, s_scalar,
                (cls == CLS_RESOLVE) ? ART_INFO_FP64_RESOLVE : 0u);
  }
}

// ============================================================== QR kernel
// FP64 Householder QR of the augmented least-squares problem
//   [sqrt(W) Phi | sqrt(W) y ; sqrt(lambda) I | 0]
// streamed in row chunks, keeping only R (with Q^T b as its last column);
// the fallback of solve_weighted_ridge's auto solver (models.py:334-357,
// _solve_augmented_ridge 374-448).  Rank-revealing pivoting (gelsy) is not
// used: the regularised problem has full column rank whenever lambda > 0.
// solver="svd" (and auto, when the QR solution is not finite) continues
// from R with the Jacobi SVD below (gelsd's minimum-norm solution).
constexpr int kQrChunk = 32;

__device__ __forceinline__ int ru(int i, int j, int pa) {  // packed upper, row-major
  return i * pa - i * (i - 1) / 2 + (j - i);
}

// SVD stage (solver="svd", or auto after a non-finite QR solution): the
// factor R is expanded in place to M = R^T, dense column-major p x p, over
// the packed R; the rotated right-hand side and the per-column scales
// follow it.
__host__ __device__ inline size_t svd_vec_off(int pmax) {
  const size_t pa = (size_t)pmax + 1;
  const size_t packed = pa * (pa + 1) / 2, dense = (size_t)pmax * pmax;
  return align16((packed > dense ? packed : dense) * 8);
}

__host__ __device__ inline size_t qr_smem(int pmax, int dmax) {
  const int pa = pmax + 1;
  size_t o = 0;
  o = align16(o + (size_t)pa * (pa + 1) / 2 * 8);   // R packed upper
  o = align16(o + (size_t)kQrChunk * pa * 8);       // V chunk
  o = align16(o + (size_t)kQrChunk * 8);            // reflector
  o = align16(o + (size_t)kQrChunk * dmax * 8);     // x chunk
  o = align16(o + (size_t)(pa + 1) * 8);            // solution
  o = align16(o + (size_t)pa * 4);                  // factor indices
  const size_t svd = svd_vec_off(pmax) + 2 * align16((size_t)pmax * 8);
  return o > svd ? o : svd;
}

// Minimum-norm least-squares solution from the triangular factor R (packed
// upper, pa = p + 1 columns, the last holding c = Q^T b) by a one-sided
// Jacobi SVD (Hestenes) of M = R^T, the LAPACK gelsd answer of
// _solve_augmented_ridge (models.py:374-448) up to rounding:
//   rotations J make the columns of M J orthogonal, M J = U' S, so
//   R = J S U'^T and  x = U' S^+ J^T c = sum_i m_i (J^T c)_i / s_i^2,
//   with s_i = ||m_i|| and singular values s_i <= eps * s_max dropped
//   (scipy's lstsq default cond = eps).  J^T c is accumulated by applying
//   every rotation to c, so J itself is never stored.
// Column pairs are visited in round-robin (circle) order, p/2 disjoint pairs
// per step, one warp per pair; sweeps stop when no pair needed a rotation
// (|m_i . m_j| <= sqrt(p) eps ||m_i|| ||m_j||) or after kSvdMaxSweeps.
// Writes the p coefficients to out (global memory: every shared byte of
// the kernel may be in use) and returns in s_res the largest and smallest
// singular value, the rank and whether a coefficient is not finite.
constexpr int kSvdMaxSweeps = 60;

__device__ void jacobi_svd_solve(double* R, int p, double* dv, double* cf, double* out, double* s_res) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = kRidgeThreads / 32;
  const int pa = p + 1;
  double* M = R;  // the same storage, expanded in place
  __shared__ int s_rot;
  for (int j = tid; j < p; j += kRidgeThreads) dv[j] = R[ru(j, p, pa)];
  __syncthreads();
  // row j of R -> column j of M, last row first: the column's slots never
  // overlap a packed row not yet moved, and c was saved above
  for (int j = p - 1; j >= 0; --j) {
    double v = 0.0;
    if (tid < p && tid >= j) v = R[ru(j, tid, pa)];
    __syncthreads();
    if (tid < p) M[(size_t)j * p + tid] = v;
    __syncthreads();
  }
  const double eps = 2.220446049250313e-16;
  const double tol = sqrt((double)p) * eps;
  const int n2 = (p + 1) & ~1;  // players of the circle schedule (one dummy when p is odd)
  for (int sweep = 0; sweep < kSvdMaxSweeps && n2 > 1; ++sweep) {
    if (tid == 0) s_rot = 0;
    __syncthreads();
    for (int step = 0; step < n2 - 1; ++step) {
      for (int q = warp; q < n2 / 2; q += nwarps) {
        int i, j;
        if (q == 0) { i = step; j = n2 - 1; }
        else { i = (step + q) % (n2 - 1); j = (step - q + (n2 - 1)) % (n2 - 1); }
        if (i >= p || j >= p) continue;
        double* mi = M + (size_t)i * p;
        double* mj = M + (size_t)j * p;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int k = lane; k < p; k += 32) {
          const double u = mi[k], v = mj[k];
          al = fma(u, u, al);
          be = fma(v, v, be);
          ga = fma(u, v, ga);
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (ga != 0.0 && fabs(ga) > tol * sqrt(al) * sqrt(be)) {
          const double zeta = (be - al) / (2.0 * ga);
          const double t = copysign(1.0, zeta) / (fabs(zeta) + hypot(1.0, zeta));
          const double c = 1.0 / sqrt(fma(t, t, 1.0)), s = c * t;
          for (int k = lane; k < p; k += 32) {
            const double u = mi[k], v = mj[k];
            mi[k] = c * u - s * v;
            mj[k] = s * u + c * v;
          }
          if (lane == 0) {
            const double u = dv[i], v = dv[j];
            dv[i] = c * u - s * v;
            dv[j] = s * u + c * v;
            s_rot = 1;
          }
        }
      }
      __syncthreads();
    }
    const int any = s_rot;
    __syncthreads();
    if (!any) break;
  }
  for (int i = warp; i < p; i += nwarps) {
    double s2 = 0.0;
    for (int k = lane; k < p; k += 32) s2 = fma(M[(size_t)i * p + k], M[(size_t)i * p + k], s2);
    s2 = warp_sum(s2);
    if (lane == 0) cf[i] = sqrt(s2);
  }
  __syncthreads();
  if (tid == 0) {
    double smax = 0.0, smin = __longlong_as_double(0x7ff0000000000000ll);
    for (int i = 0; i < p; ++i) { smax = fmax(smax, cf[i]); smin = fmin(smin, cf[i]); }
    int rank = 0;
    for (int i = 0; i < p; ++i) {
      const double si = cf[i];
      const bool keep = si > eps * smax;
      rank += keep ? 1 : 0;
      cf[i] = keep ? dv[i] / (si * si) : 0.0;
    }
    s_res[0] = smax;
    s_res[1] = smin;
    s_res[2] = (double)rank;
  }
  __syncthreads();
  int nonfinite = 0;
  for (int k = tid; k < p; k += kRidgeThreads) {
    double x = 0.0;
    for (int i = 0; i < p; ++i) x = fma(M[(size_t)i * p + k], cf[i], x);
    nonfinite |= !isfinite(x);
    out[k] = x;
  }
  nonfinite = __syncthreads_or(nonfinite);
  if (tid == 0) s_res[3] = nonfinite ? 1.0 : 0.0;
  __syncthreads();
}

__global__ void __launch_bounds__(kRidgeThreads) ridge_qr_kernel(RidgeArgs a, RidgeLists L) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  __shared__ double s_tau;
  __shared__ double s_svd[4];
  const int pa_max = a.pmax + 1;
  double* R = (double*)smem;
  double* V = (double*)(smem + align16((size_t)pa_max * (pa_max + 1) / 2 * 8));
  double* vb = V + align16((size_t)kQrChunk * pa_max * 8) / 8;
  double* xs = vb + align16((size_t)kQrChunk * 8) / 8;
  double* sol = xs + align16((size_t)kQrChunk * a.dmax * 8) / 8;
  int16_t* fidx = (int16_t*)(sol + align16((size_t)(pa_max + 1) * 8) / 8);
  const int tid = threadIdx.x, lane = tid & 31;
  const int count = L.count[CLS_QR];
  for (;;) {
    if (tid == 0) s_item = atomicAdd(&L.cursor[CLS_QR], 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= count) break;
    const int k = L.list[(int64_t)CLS_QR * a.K + item];
    const RidgeItem it = load_item(a, k);
    const int p = it.p, pa = p + 1, d = it.d;
    const double lam = L.lambda[k];
    for (int e = tid; e < pa * (pa + 1) / 2; e += kRidgeThreads) R[e] = 0.0;
    for (int f = tid; f < p; f += kRidgeThreads) {
      int fa_, fb_;
      feature_factors(d, it.kind, f, fa_, fb_);
      fidx[2 * f] = (int16_t)fa_;
      fidx[2 * f + 1] = (int16_t)fb_;
    }
    __syncthreads();
    const int64_t n_lam = (lam > 0.0) ? p : 0;
    const int64_t total = it.n + n_lam;
    for (int64_t c0 = 0; c0 < total; c0 += kQrChunk) {
      const int rows = (int)min((int64_t)kQrChunk, total - c0);
      // build V rows
      const int64_t data_rows = max((int64_t)0, min((int64_t)rows, it.n - c0));
      for (int e = tid; e < data_rows * d; e += kRidgeThreads)
        xs[e] = a.x[it.xoff + c0 * d + e];
      __syncthreads();
      for (int e = tid; e < rows * pa; e += kRidgeThreads) {
        const int r = e / pa, f = e - r * pa;
        const int64_t g = c0 + r;
        double v;
        if (g < it.n) {
          double wv = a.w ? a.w[it.r0 + g] : 1.0;
          double sw = sqrt(fmax(wv, a.weight_floor));
          if (f == p) v = sw * a.y[it.r0 + g];
          else {
            const int ia = fidx[2 * f], ib = fidx[2 * f + 1];
            const double* xr = xs + (int64_t)r * d;
            v = sw * ((ia < 0 ? 1.0 : xr[ia]) * (ib < 0 ? 1.0 : xr[ib]));
          }
        } else {
          const int64_t li = g - it.n;  // ridge row li
          v = (f == li) ? sqrt(lam) : 0.0;
        }
        V[r * pa + f] = v;
      }
      __syncthreads();
      for (int j = 0; j < p; ++j) {
        if (tid < 32) {
          double sig = 0.0;
          for (int r = lane; r < rows; r += 32) sig += V[r * pa + j] * V[r * pa + j];
          sig = warp_sum(sig);
          const double x0 = R[ru(j, j, pa)];
          double tau = 0.0, scale = 0.0, beta = x0;
          if (sig > 0.0) {
            const double mu = sqrt(x0 * x0 + sig);
            beta = -copysign(mu, x0);
            tau = (beta - x0) / beta;
            scale = 1.0 / (x0 - beta);
          }
          for (int r = lane; r < rows; r += 32) vb[r] = V[r * pa + j] * scale;
          if (lane == 0) {
            s_tau = tau;
            R[ru(j, j, pa)] = beta;
          }
        }
        __syncthreads();
        const double tau = s_tau;
        if (tau != 0.0) {
          for (int col = j + 1 + tid; col < pa; col += kRidgeThreads) {
            double s = R[ru(j, col, pa)];
            for (int r = 0; r < rows; ++r) s = fma(vb[r], V[r * pa + col], s);
            s *= tau;
            R[ru(j, col, pa)] -= s;
            for (int r = 0; r < rows; ++r) V[r * pa + col] = fma(-s, vb[r], V[r * pa + col]);
          }
        }
        __syncthreads();
      }
    }
    bool use_svd = a.solver == ART_SOLVER_SVD;
    if (!use_svd) {
      // back substitution R beta = c, c = R[:, p]
      if (tid < 32) {
        for (int i = lane; i < p; i += 32) sol[i] = R[ru(i, p, pa)];
        __syncwarp();
        for (int j = p - 1; j >= 0; --j) {
          if (lane == 0) sol[j] = sol[j] / R[ru(j, j, pa)];
          __syncwarp();
          const double bj = sol[j];
          for (int i = lane; i < j; i += 32) sol[i] -= R[ru(i, j, pa)] * bj;
          __syncwarp();
        }
      }
      __syncthreads();
      int nonfinite = 0;
      for (int i = tid; i < p; i += kRidgeThreads) nonfinite |= !isfinite(sol[i]);
      nonfinite = __syncthreads_or(nonfinite);
      // auto: a non-finite QR solution is re-solved by the SVD (models.py:426-438)
      if (nonfinite && a.solver == ART_SOLVER_AUTO) {
        use_svd = true;
      } else {
        for (int i = tid; i < p; i += kRidgeThreads) a.beta[(int64_t)k * a.beta_stride + i] = sol[i];
        if (tid == 0) a.status[k] = nonfinite ? -3 : 0;
        __syncthreads();
        continue;
      }
    }
    // SVD path: the vectors live past the expanded M (which covers the QR
    // work arrays, sol included)
    double* dv = (double*)(smem + svd_vec_off(a.pmax));
    double* cf = dv + align16((size_t)a.pmax * 8) / 8;
    jacobi_svd_solve(R, p, dv, cf, a.beta + (int64_t)k * a.beta_stride, s_svd);
    if (tid == 0) {
      a.status[k] = s_svd[3] != 0.0 ? -3 : 0;
      const double smax = s_svd[0], smin = s_svd[1];
      if (a.cond) a.cond[k] = smin > 0.0 ? smax / smin : __longlong_as_double(0x7ff0000000000000ll);
      if (a.info)
        a.info[k] = a.info[k] | ART_INFO_SVD | ((uint32_t)s_svd[2] << ART_INFO_RANK_SHIFT);
    }
    __syncthreads();
  }
}

// ================================================================== host
static int g_sm_count[64];

int device_sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!g_sm_count[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    g_sm_count[dev] = v > 0 ? v : 148;
  }
  return g_sm_count[dev];
}

struct WsLayout {
  size_t off_count, off_cursor, off_hist, off_start, off_err, off_lambda, off_list, header,
      total;
};
static constexpr WsLayout ws_layout(int64_t K) {
  WsLayout w{};
  size_t o = 0;
  w.off_count = o; o += kClasses * 4;
  w.off_cursor = o; o += kClasses * 4;
  w.off_hist = o; o += kPlanClasses * kBuckets * 4;
  w.off_start = o; o += kPlanClasses * kBuckets * 4;
  w.off_err = o; o += 16;
  w.header = o;  // zeroed every call
  o = (o + 255) & ~(size_t)255;
  w.off_lambda = o; o += (size_t)K * 8;
  o = (o + 255) & ~(size_t)255;
  w.off_list = o; o += (size_t)kClasses * K * 4;
  w.total = (o + 255) & ~(size_t)255;
  return w;
}

template <typename Kern>
static int launch_persistent(Kern kern, size_t smem, int64_t max_items, cudaStream_t s,
                             RidgeArgs a, RidgeLists L, int cls, int pcap, const char* name) {
  if (smem > 227 * 1024) {
    set_error("%s: shared memory %zu bytes exceeds the 227 KB limit", name, smem);
    return ART_E_UNSUPPORTED;
  }
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("%s: cannot reserve %zu bytes of shared memory", name, smem);
    return ART_E_UNSUPPORTED;
  }
  const int occ = resident_ctas((const void*)kern, kRidgeThreads, smem);
  int64_t grid = (int64_t)device_sm_count() * occ;
  if (grid > max_items) grid = max_items;
  if (grid < 1) grid = 1;
  prof_begin(name, s);
  kern<<<(unsigned)grid, kRidgeThreads, smem, s>>>(a, L, cls, pcap);
  prof_end(s);
  count_launch();
  return check_launch(name);
}

}  // namespace art

using namespace art;

extern "C" size_t art_ridge_workspace_size(int64_t count, int32_t max_features) {
  (void)max_features;
  if (count < 0) return 0;
  return ws_layout(count).total;
}

static int ridge_entry(const ArtRidgeProblem* pr, const ArtRidgeResult* res, float* gram_out,
                       int64_t gram_stride, void* workspace, size_t ws_bytes, art_stream_t stream) {
  if (!pr || !res) { set_error("art_ridge_batched: null problem/result"); return ART_E_INVALID; }
  const int64_t K = pr->seg.count;
  if (K < 0) { set_error("art_ridge_batched: negative count"); return ART_E_INVALID; }
  if (K == 0) return ART_OK;
  if (!pr->seg.row_offsets || !pr->seg.x_offsets || !pr->seg.dims || !pr->seg.features ||
      !pr->x || !pr->y || !pr->ridge || !res->beta || !res->status) {
    set_error("art_ridge_batched: null device pointer");
    return ART_E_INVALID;
  }
  if (pr->max_features < 1 || pr->max_features > ART_MAX_FEATURES) {
    set_error("art_ridge_batched: max_features %d outside [1, %d]", pr->max_features,
              ART_MAX_FEATURES);
    return ART_E_UNSUPPORTED;
  }
  if (res->beta_stride < pr->max_features) {
    set_error("art_ridge_batched: beta_stride %lld < max_features %d",
              (long long)res->beta_stride, pr->max_features);
    return ART_E_INVALID;
  }
  if (pr->solver != ART_SOLVER_NORMAL && pr->solver != ART_SOLVER_AUTO &&
      pr->solver != ART_SOLVER_QR && pr->solver != ART_SOLVER_SVD) {
    set_error("art_ridge_batched: unknown solver %d", pr->solver);
    return ART_E_INVALID;
  }
  if (pr->precision != ART_PRECISION_FP64 && pr->precision != ART_PRECISION_MIXED) {
    set_error("art_ridge_batched: unknown precision %d", pr->precision);
    return ART_E_INVALID;
  }
  if (!(pr->auto_rcond_threshold > 0.0 && pr->auto_rcond_threshold <= 1.0)) {
    set_error("auto_rcond_threshold must satisfy 0 < value <= 1.");
    return ART_E_INVALID;
  }
  if (!(pr->weight_floor >= 0.0)) {
    set_error("art_ridge_batched: weight_floor must be nonnegative");
    return ART_E_INVALID;
  }
  const WsLayout wl = ws_layout(K);
  if (!workspace || ws_bytes < wl.total) {
    set_error("art_ridge_batched: workspace %zu bytes < required %zu", ws_bytes, wl.total);
    return ART_E_WORKSPACE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaGetLastError();  // clear a stale, non-sticky error left by an earlier runtime call
  unsigned char* ws = (unsigned char*)workspace;
  RidgeArgs a;
  a.K = K;
  a.row_offsets = pr->seg.row_offsets;
  a.x_offsets = pr->seg.x_offsets;
  a.dims = pr->seg.dims;
  a.features = pr->seg.features;
  a.x = pr->x; a.y = pr->y; a.w = pr->w; a.ridge = pr->ridge;
  a.weight_floor = pr->weight_floor;
  a.solver = pr->solver;
  a.precision = pr->precision;
  // The tensor-core form stages rows of at most ART_MAX_DIM inputs; wider
  // explicit designs are solved by the FP64 form.
  if (a.precision == ART_PRECISION_MIXED && pr->max_dim > ART_MAX_DIM) a.precision = ART_PRECISION_FP64;
  a.rcond_threshold = pr->auto_rcond_threshold;
  a.pmax = pr->max_features;
  a.dmax = pr->max_dim > 0 ? std::min(pr->max_dim, pr->max_features) : pr->max_features;
  if (a.dmax > ART_MAX_FEATURES) a.dmax = ART_MAX_FEATURES;
  a.beta = res->beta; a.beta_stride = res->beta_stride;
  a.ridge_eff = res->ridge_effective; a.cond = res->cond_estimate;
  a.status = res->status; a.info = res->info;
  a.options = pr->options;
  a.tensor_min_p = pr->tensor_min_features > 0 ? std::max(pr->tensor_min_features, kTensorMinP) : kTensorMinP;
  if (gram_out) a.tensor_min_p = kTensorMinP;
  a.gram_out = gram_out;
  a.gram_stride = gram_stride;
  if (gram_out) a.precision = ART_PRECISION_MIXED;
  RidgeLists L;
  L.count = (int32_t*)(ws + wl.off_count);
  L.cursor = (int32_t*)(ws + wl.off_cursor);
  L.hist = (int32_t*)(ws + wl.off_hist);
  L.start = (int32_t*)(ws + wl.off_start);
  L.err = (int32_t*)(ws + wl.off_err);
  L.lambda = (double*)(ws + wl.off_lambda);
  L.list = (int32_t*)(ws + wl.off_list);
  if (cudaMemsetAsync(ws, 0, wl.header, s) != cudaSuccess) return check_launch("memset");
  const unsigned pg = (unsigned)((K + 255) / 256);
  prof_begin("ridge_plan", s);
  ridge_plan_hist<<<pg, 256, 0, s>>>(a, L);
  ridge_plan_scan<<<1, 32 * kPlanClasses, 0, s>>>(L);
  ridge_plan_scatter<<<pg, 256, 0, s>>>(a, L);
  prof_end(s);
  count_launch();
  count_launch();
  count_launch();
  int rc = check_launch("ridge plan");
  if (rc) return rc;
  if (a.precision == ART_PRECISION_MIXED) {
    rc = launch_ridge_tensor(a, L, s);
    if (rc) return rc;
  }
  if (gram_out) return ART_OK;
  rc = launch_ridge_warp(a, L, s);
  if (rc) return rc;
  if (a.pmax + 1 > kWarpMaxAug) {
    const int pcap = std::min(a.pmax, kSmallMaxAug - 1);
    const size_t sm = fp64_layout(pcap, a.dmax, 4, 64).total;
    rc = launch_persistent(ridge_fp64_kernel<4, 64>, sm, K, s, a, L, CLS_SMALL, pcap,
                           "ridge_fp64<4>");
    if (rc) return rc;
  }
  if (a.pmax + 1 > kSmallMaxAug || a.precision == ART_PRECISION_MIXED) {
    const size_t sm = fp64_layout(a.pmax, a.dmax, 8, 32).total;
    rc = launch_persistent(ridge_fp64_kernel<8, 32>, sm, K, s, a, L, CLS_LARGE, a.pmax,
                           "ridge_fp64<8>");
    if (rc) return rc;
    if (a.precision == ART_PRECISION_MIXED) {
      rc = launch_persistent(ridge_fp64_kernel<8, 32>, sm, K, s, a, L, CLS_RESOLVE, a.pmax,
                             "ridge_fp64<8> resolve");
      if (rc) return rc;
    }
  }
  if (a.solver == ART_SOLVER_AUTO || a.solver == ART_SOLVER_QR || a.solver == ART_SOLVER_SVD) {
    const size_t sm = qr_smem(a.pmax, a.dmax);
    if (sm > 227 * 1024) {
      set_error("ridge_qr: shared memory %zu bytes exceeds the 227 KB limit", sm);
      return ART_E_UNSUPPORTED;
    }
    if (cudaFuncSetAttribute(ridge_qr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
        cudaSuccess) {
      cudaGetLastError();
      set_error("ridge_qr: cannot reserve %zu bytes of shared memory", sm);
      return ART_E_UNSUPPORTED;
    }
    int64_t grid = std::min<int64_t>(K, device_sm_count());
    prof_begin("ridge_qr", s);
    ridge_qr_kernel<<<(unsigned)grid, kRidgeThreads, sm, s>>>(a, L);
    prof_end(s);
    count_launch();
    rc = check_launch("ridge_qr");
    if (rc) return rc;
  }
  return ART_OK;
}

extern "C" int art_ridge_batched(const ArtRidgeProblem* pr, const ArtRidgeResult* res,
                                 void* workspace, size_t ws_bytes, art_stream_t stream) {
  return ridge_entry(pr, res, nullptr, 0, workspace, ws_bytes, stream);
}

// Fixed scratch of art_ridge_batched_noalloc: the workspace layout for
// ART_RIDGE_NOALLOC_MAX_COUNT systems (about 1.8 MiB), a file-scope device
// array so that the call itself allocates nothing.
static constexpr size_t kNoallocBytes = ws_layout(ART_RIDGE_NOALLOC_MAX_COUNT).total;
static __device__ __align__(256) unsigned char g_ridge_noalloc_ws[kNoallocBytes];
// Device address of the array per device ordinal, resolved on a device's
// first call.  Host threads may race on the first call; each resolves the
// same address, and the release/acquire pair publishes it.  The cache
// assumes the device's primary context (the one the runtime API uses): after
// cudaDeviceReset the module is reloaded and the address may change, so a
// caller that resets a device must not call this entry point again in the
// same process.
static std::atomic<void*> g_noalloc_addr[64];

extern "C" size_t art_ridge_noalloc_scratch_bytes(void) { return kNoallocBytes; }

extern "C" int art_ridge_batched_noalloc(const ArtRidgeProblem* pr, const ArtRidgeResult* res,
                                         art_stream_t stream) {
  if (pr && pr->seg.count > ART_RIDGE_NOALLOC_MAX_COUNT) {
    set_error("art_ridge_batched_noalloc: %lld systems exceed the fixed scratch limit of %d",
              (long long)pr->seg.count, ART_RIDGE_NOALLOC_MAX_COUNT);
    return ART_E_UNSUPPORTED;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    set_error("art_ridge_batched_noalloc: no usable current device");
    return ART_E_DEVICE;
  }
  // Resolved once per device; the first call on a device may load the module.
  void* addr = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!addr) {
    if (cudaGetSymbolAddress(&addr, g_ridge_noalloc_ws) != cudaSuccess || !addr) {
      cudaGetLastError();
      set_error("art_ridge_batched_noalloc: cannot resolve the scratch address");
      return ART_E_LAUNCH;
    }
    g_noalloc_addr[dev].store(addr, std::memory_order_release);
  }
  return ridge_entry(pr, res, nullptr, 0, addr, kNoallocBytes, stream);
}

extern "C" int art_ridge_gram(const ArtRidgeProblem* pr, float* gram, int64_t gram_stride,
                              int32_t* status, void* workspace, size_t ws_bytes,
                              art_stream_t stream) {
  if (!pr || !gram || !status) { set_error("art_ridge_gram: null argument"); return ART_E_INVALID; }
  if (pr->max_dim > ART_MAX_DIM || pr->max_features > ART_MAX_FEATURES) {
    set_error("art_ridge_gram: max_dim <= %d and max_features <= %d required", ART_MAX_DIM,
              ART_MAX_FEATURES);
    return ART_E_UNSUPPORTED;
  }
  if (gram_stride < (int64_t)pr->max_features * (pr->max_features + 1) / 2) {
    set_error("art_ridge_gram: gram_stride below p(p+1)/2");
    return ART_E_INVALID;
  }
  // beta is not written by a Gram-only call; any non-null pointer satisfies validation
  ArtRidgeResult res{};
  res.beta = (double*)gram;
  res.beta_stride = pr->max_features;
  res.status = status;
  return ridge_entry(pr, &res, gram, gram_stride, workspace, ws_bytes, stream);
}
