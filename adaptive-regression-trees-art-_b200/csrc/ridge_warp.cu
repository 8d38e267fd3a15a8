// ridge_warp.cu -- FP64 weighted ridge for narrow systems, one warp per system.
//
// Systems with an augmented width p + 1 <= kWarpMaxAug (affine models up to
// d = 22, degree-2 models up to d = 5) carry too little arithmetic per row
// to keep a 256-thread CTA busy between block barriers, and the whole class
// is HBM-bound (1.4-2.4 flop per input byte at FP64).  Here every warp works
// alone: it streams its system's rows through two shared-memory stages by
// 1-D bulk copies (issued by lane 0, completed on a per-warp mbarrier), so
// there is no block-wide barrier after set-up.
//
// Per batch of 32 rows:
//   1. lane r forms the augmented feature row sqrt(q_r) [phi(x_r), y_r]
//      (q = max(w, floor), models.py:250-262) into a row-major tile P;
//   2. the lanes, split into G row groups x NB lower-triangular 4x4 blocks
//      of the augmented Gram, accumulate their block over the rows of their
//      group with FP64 FMAs (two 16-byte loads per operand block).
// The row groups are summed in a fixed order, then one warp finishes the
// system exactly as the CTA form does (trace-scaled ridge, Cholesky, solve,
// condition estimate and the auto-solver policy of models.py:268-371).
#include <algorithm>

#include "ridge.cuh"

namespace art {
namespace {

constexpr int kWarpThreads = 128;             // 4 independent warps per CTA
constexpr int kWarpsPerCta = kWarpThreads / 32;
constexpr int kWRows = 32;                    // rows per batch (one per lane)
constexpr int kWPad = kWarpMaxAug;            // padded augmented width (multiple of 4)
constexpr int kWLdr = kWPad + 2;              // row stride of P (even: 16-byte rows; 26 = 10 mod 16 spreads rows over banks)

__host__ __device__ inline size_t wa16(size_t v) { return (v + 15) & ~(size_t)15; }

struct WarpLayout {
  size_t x[2], y[2], w[2], P, G, vec, fidx, bars, per_warp;
};

__host__ __device__ inline WarpLayout warp_layout(int dw) {
  WarpLayout L;
  size_t o = 0;
  for (int s = 0; s < 2; ++s) {
    L.x[s] = o; o = wa16(o + (size_t)kWRows * dw * 8 + 16);
    L.y[s] = o; o = wa16(o + (size_t)kWRows * 8 + 16);
    L.w[s] = o; o = wa16(o + (size_t)kWRows * 8 + 16);
  }
  L.P = o; o = wa16(o + (size_t)kWRows * kWLdr * 8);
  L.G = o; o = wa16(o + (size_t)kWPad * (kWPad + 1) / 2 * 8);
  L.vec = o; o = wa16(o + (size_t)3 * (kWPad + 1) * 8);
  L.fidx = o; o = wa16(o + (size_t)kWPad * 2 * 2);
  L.bars = o; o = wa16(o + 2 * 8);
  L.per_warp = (o + 127) & ~(size_t)127;
  return L;
}

__device__ __forceinline__ void warp_issue(const RidgeArgs& a, const RidgeItem& it, int64_t c,
                                           unsigned char* base, const WarpLayout& lay, int st,
                                           uint64_t* bar) {
  const int64_t rr = c * kWRows;
  const int rows = (int)min((int64_t)kWRows, it.n - rr);
  Granules gx = granules(a.x + it.xoff + rr * it.d, (uint64_t)rows * it.d * 8);
  Granules gy = granules(a.y + it.r0 + rr, (uint64_t)rows * 8);
  Granules gw = a.w ? granules(a.w + it.r0 + rr, (uint64_t)rows * 8) : Granules{nullptr, 0, 0};
  mbar_arrive_expect_tx(bar, gx.bytes + gy.bytes + gw.bytes);
  bulk_g2s(base + lay.x[st], gx.base, gx.bytes, bar);
  bulk_g2s(base + lay.y[st], gy.base, gy.bytes, bar);
  if (a.w) bulk_g2s(base + lay.w[st], gw.base, gw.bytes, bar);
}

// Packed lower Cholesky by one warp (right-looking, column at a time).
// Returns 0 or the 1-based index of the first non-positive pivot.
__device__ int warp_chol_packed(double* A, int p) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < p; ++j) {
    __syncwarp();
    const double djj = A[pk(j, j)];
    if (!(djj > 0.0) || !isfinite(djj)) return j + 1;
    const double l = sqrt(djj);
    __syncwarp();
    if (lane == 0) A[pk(j, j)] = l;
    for (int i = j + 1 + lane; i < p; i += 32) A[pk(i, j)] = A[pk(i, j)] / l;
    __syncwarp();
    const int m = p - j - 1;
    const int E = m * (m + 1) / 2;
    for (int e = lane; e < E; e += 32) {
      const int ii = tile_row(e), kk = e - ii * (ii + 1) / 2;
      const int i = j + 1 + ii, k = j + 1 + kk;
      A[pk(i, k)] -= A[pk(i, j)] * A[pk(k, j)];
    }
  }
  __syncwarp();
  return 0;
}

__device__ void warp_write_failed(const RidgeArgs& a, int k, int p, int32_t status, double lam,
                                  uint32_t info) {
  const int lane = threadIdx.x & 31;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  for (int i = lane; i < p; i += 32) a.beta[(int64_t)k * a.beta_stride + i] = nan;
  if (lane == 0) {
    a.status[k] = status;
    if (a.ridge_eff) a.ridge_eff[k] = lam;
    if (a.cond) a.cond[k] = nan;
    if (a.info) a.info[k] = info;
  }
}

// The finish step of the CTA form (finish_fp64), by one warp.
__device__ void warp_finish(const RidgeArgs& a, const RidgeLists& L, int k, const RidgeItem& it,
                            double* G, int bad, double* vec) {
  const int lane = threadIdx.x & 31, p = it.p;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const double inf = __longlong_as_double(0x7ff0000000000000ll);
  double tr = 0.0;
  for (int i = 0; i < p; ++i) tr += G[pk(i, i)];
  const double lam = it.ridge * tr / p;
  if (lane == 0) L.lambda[k] = lam;
  if (bad) {
    warp_write_failed(a, k, p, (bad & 2) ? -1 : -2, lam, 0u);
    return;
  }
  if (a.solver == ART_SOLVER_QR || a.solver == ART_SOLVER_SVD) {
    if (lane == 0) {
      if (a.ridge_eff) a.ridge_eff[k] = lam;
      if (a.cond) a.cond[k] = nan;
      if (a.info) a.info[k] = a.solver == ART_SOLVER_SVD ? 0u : ART_INFO_QR_FALLBACK;
      a.status[k] = 0;
      push_list(L, a.K, CLS_QR, k);
    }
    return;
  }
  __syncwarp();
  for (int i = lane; i < p; i += 32) G[pk(i, i)] += lam;
  __syncwarp();
  const bool want_cond = (a.cond != nullptr) || (a.solver == ART_SOLVER_AUTO);
  const double an = want_cond ? warp_sym_norm1(G, p) : 0.0;
  const int fail = warp_chol_packed(G, p);
  if (fail) {
    if (a.solver == ART_SOLVER_AUTO) {
      if (lane == 0) {
        if (a.ridge_eff) a.ridge_eff[k] = lam;
        if (a.cond) a.cond[k] = inf;
        if (a.info) a.info[k] = ART_INFO_QR_FALLBACK | ART_INFO_CHOLESKY_FAILED;
        a.status[k] = 0;
        push_list(L, a.K, CLS_QR, k);
      }
      return;
    }
    warp_write_failed(a, k, p, fail, lam, 0u);
    return;
  }
  double* z = vec;
  double* v = vec + (kWPad + 1);
  double* sg = vec + 2 * (kWPad + 1);
  for (int i = lane; i < p; i += 32) z[i] = G[pk(p, i)];  // h
  __syncwarp();
  warp_forward<double, double>(G, z, p);
  warp_backward<double, double>(G, z, p);
  uint32_t info = 0;
  double cond = nan;
  if (want_cond) {
    const double est = warp_inv_norm1_estimate<double>(G, p, v, sg);
    double rcond = (est > 0.0 && isfinite(est) && an > 0.0) ? 1.0 / (an * est) : 0.0;
    if (rcond > 0.0 && isfinite(rcond)) {
      cond = sqrt(1.0 / fmin(rcond, 1.0));
    } else {
      rcond = 0.0;
      cond = inf;
      info |= ART_INFO_COND_FAILED;
    }
    if (a.solver == ART_SOLVER_AUTO && rcond < a.rcond_threshold) {
      if (lane == 0) {
        if (a.ridge_eff) a.ridge_eff[k] = lam;
        if (a.cond) a.cond[k] = cond;
        if (a.info) a.info[k] = info | ART_INFO_QR_FALLBACK | ART_INFO_RCOND_BELOW;
        a.status[k] = 0;
        push_list(L, a.K, CLS_QR, k);
      }
      return;
    }
  }
  __syncwarp();
  int nonfinite = 0;
  for (int i = lane; i < p; i += 32) {
    const double b = z[i];
    nonfinite |= !isfinite(b);
    a.beta[(int64_t)k * a.beta_stride + i] = b;
  }
  nonfinite = __any_sync(0xffffffffu, nonfinite);
  if (lane == 0) {
    a.status[k] = nonfinite ? -3 : 0;
    if (a.ridge_eff) a.ridge_eff[k] = lam;
    if (a.cond) a.cond[k] = cond;
    if (a.info) a.info[k] = info;
  }
}

__global__ void __launch_bounds__(kWarpThreads) ridge_warp_kernel(RidgeArgs a, RidgeLists L, int dw) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const WarpLayout lay = warp_layout(dw);
  unsigned char* base = smem + (size_t)warp * lay.per_warp;
  double* P = (double*)(base + lay.P);
  double* G = (double*)(base + lay.G);
  double* vec = (double*)(base + lay.vec);
  int16_t* fidx = (int16_t*)(base + lay.fidx);
  uint64_t* bars = (uint64_t*)(base + lay.bars);
  if (lane == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncwarp();
  uint32_t uses[2] = {0u, 0u};
  const int count = L.count[CLS_WARP];
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(&L.cursor[CLS_WARP], 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= count) break;
    const int k = L.list[(int64_t)CLS_WARP * a.K + item];
    const RidgeItem it = load_item(a, k);
    const int p = it.p, pa = p + 1, d = it.d;
    const int PW = (pa + 3) & ~3;
    const int nb = PW >> 2, NB = nb * (nb + 1) / 2;
    const int NG = 32 / NB;  // row groups
    for (int f = lane; f < PW; f += 32) {
      int fa_, fb_;
      if (f < p) feature_factors(d, it.kind, f, fa_, fb_);
      else if (f == p) { fa_ = -2; fb_ = -1; }
      else { fa_ = -3; fb_ = -1; }
      fidx[2 * f] = (int16_t)fa_;
      fidx[2 * f + 1] = (int16_t)fb_;
    }
    const bool mine = lane < NG * NB;
    const int blk = mine ? lane % NB : 0, grp = mine ? lane / NB : 0;
    const int I = tile_row(blk), J = blk - I * (I + 1) / 2;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    int bad = 0;
    bool timed_out = false;
    int64_t timed_c = 0;
    const int64_t nb_batches = (it.n + kWRows - 1) / kWRows;
    if (lane == 0)
      for (int64_t c = 0; c < min((int64_t)2, nb_batches); ++c)
        warp_issue(a, it, c, base, lay, (int)c, &bars[c]);
    __syncwarp();
    for (int64_t c = 0; c < nb_batches; ++c) {
      const int st = (int)(c & 1);
      const bool ok = mbar_wait(&bars[st], uses[st] & 1);
      if (!__all_sync(0xffffffffu, ok)) { timed_out = true; timed_c = c; break; }
      uses[st]++;
      const int rows = (int)min((int64_t)kWRows, it.n - c * kWRows);
      const double* xs = (const double*)(base + lay.x[st] +
                                         (((uintptr_t)(a.x + it.xoff + c * kWRows * d)) & 15));
      const double* ys = (const double*)(base + lay.y[st] + (((uintptr_t)(a.y + it.r0 + c * kWRows)) & 15));
      const double* ws = a.w ? (const double*)(base + lay.w[st] +
                                               (((uintptr_t)(a.w + it.r0 + c * kWRows)) & 15))
                             : nullptr;
      // 1. lane r forms row r of P (zeros past the last row).  Lane r starts
      // its walk over the inputs and features at an offset of r, so the
      // lanes' strided row accesses spread over the shared-memory banks.
      {
        const int r = lane;
        double* pr = P + r * kWLdr;
        if (r < rows) {
          const double* xr = xs + r * d;
          const int j0 = r % d;
          for (int t = 0, j = j0; t < d; ++t, j = (j + 1 == d) ? 0 : j + 1) bad |= isfinite(xr[j]) ? 0 : 1;
          const double yv = ys[r];
          bad |= isfinite(yv) ? 0 : 1;
          const double wv = ws ? ws[r] : 1.0;
          if (!(wv >= 0.0) || !isfinite(wv)) bad |= 2;
          const double sq = sqrt(fmax(wv, a.weight_floor));
          const int f0 = r % PW;
          for (int t = 0, f = f0; t < PW; ++t, f = (f + 1 == PW) ? 0 : f + 1) {
            const int ia = fidx[2 * f], ib = fidx[2 * f + 1];
            double v;
            if (ia == -3) v = 0.0;
            else if (ia == -2) v = sq * yv;
            else v = sq * ((ia < 0 ? 1.0 : xr[ia]) * (ib < 0 ? 1.0 : xr[ib]));
            pr[f] = v;
          }
        } else {
          for (int f = 0; f < PW; ++f) pr[f] = 0.0;
        }
      }
      __syncwarp();
      if (lane == 0 && c + 2 < nb_batches) warp_issue(a, it, c + 2, base, lay, st, &bars[st]);
      // 2. block accumulation over this group's rows
      if (mine) {
        for (int j = grp; j < rows; j += NG) {
          const double* pr = P + j * kWLdr;
          const double2 a01 = *(const double2*)(pr + 4 * I);
          const double2 a23 = *(const double2*)(pr + 4 * I + 2);
          const double2 b01 = *(const double2*)(pr + 4 * J);
          const double2 b23 = *(const double2*)(pr + 4 * J + 2);
          const double av[4] = {a01.x, a01.y, a23.x, a23.y};
          const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fma(av[i], bv[jj], acc[i][jj]);
        }
      }
      __syncwarp();
    }
    if (timed_out) {
      if (lane == 0) {
        atomicExch(L.err, 1);
        a.status[k] = -5;
        // bounded waits for this warp's own copies still in flight
        for (int64_t c2 = timed_c; c2 < min(timed_c + 2, nb_batches); ++c2) {
          const int s2 = (int)(c2 & 1);
          mbar_wait(&bars[s2], uses[s2] & 1);
          uses[s2]++;
        }
      }
      return;  // this warp's barrier phases are no longer consistent
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    // row groups summed in order into the packed augmented Gram
    double* part = P;  // [group][block][16]
    if (mine) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) part[(grp * NB + blk) * 16 + i * 4 + jj] = acc[i][jj];
    }
    __syncwarp();
    for (int e = lane; e < NB * 16; e += 32) {
      const int b = e >> 4, ij = e & 15;
      const int bi = tile_row(b), bj = b - bi * (bi + 1) / 2;
      const int r = 4 * bi + (ij >> 2), cc = 4 * bj + (ij & 3);
      double s = 0.0;
      for (int g = 0; g < NG; ++g) s += part[(g * NB + b) * 16 + ij];
      if (r < pa && cc <= r) G[pk(r, cc)] = s;
    }
    __syncwarp();
    warp_finish(a, L, k, it, G, bad, vec);
    __syncwarp();
  }
}

}  // namespace

size_t warp_smem_bytes(int dmax) {
  const int dw = std::min(dmax, kWarpMaxAug - 1);
  return warp_layout(dw).per_warp * kWarpsPerCta;
}

int launch_ridge_warp(const RidgeArgs& a, const RidgeLists& L, cudaStream_t s) {
  const int dw = std::min(a.dmax, kWarpMaxAug - 1);
  const size_t smem = warp_smem_bytes(a.dmax);
  if (cudaFuncSetAttribute(ridge_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("ridge_warp: cannot reserve %zu bytes of shared memory", smem);
    return ART_E_UNSUPPORTED;
  }
  const int occ = resident_ctas((const void*)ridge_warp_kernel, kWarpThreads, smem);
  int64_t grid = (int64_t)device_sm_count() * occ;
  const int64_t need = (a.K + kWarpsPerCta - 1) / kWarpsPerCta;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  prof_begin("ridge_warp", s);
  ridge_warp_kernel<<<(unsigned)grid, kWarpThreads, smem, s>>>(a, L, dw);
  prof_end(s);
  count_launch();
  return check_launch("ridge_warp");
}

}  // namespace art
