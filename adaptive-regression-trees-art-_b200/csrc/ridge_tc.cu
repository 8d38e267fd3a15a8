// ridge_tc.cu -- mixed-precision weighted ridge on the 5th-generation tensor
// cores (sm_100a tcgen05), for systems with 33 <= p <= 160 features.
//
// Per system (one CTA, persistent work queue over the CLS_TENSOR list):
//  1. Rows stream into shared memory by 1-D bulk copies (2 stages of 32 rows).
//     256 threads generate v = sqrt(q) * phi(x) for every feature and row,
//     split it into TF32 hi + lo parts (hi = rna(v), lo = rna(v - hi): about
//     22 significant bits together) and store both in the K-major
//     core-matrix layout (8 rows x 16 bytes per core matrix, no swizzle).
//     The same threads accumulate the FP64 h = sum phi (q y) and
//     diag(G) = sum (sqrt(q) phi)^2 (for the trace-scaled ridge,
//     models.py:271), one rounding per term.
//  2. One thread issues tcgen05.mma kind::tf32 (TF32 x TF32 -> FP32 in TMEM):
//     G' = Hi Hi^T + Hi Lo^T + Lo Hi^T with M = 128 feature rows per tile
//     (tile 1: features 0..127 x 0..P16-1; tile 2 covers features >= 128),
//     committed to an mbarrier per stage so operand buffers recycle.
//  3. The FP32 Gram is drained from TMEM (tcgen05.ld 32x32b) into shared
//     memory every kDrainChunks chunks, its diagonal replaced by the exact
//     FP64 diag + lambda, and factored by an FP32 Cholesky; the factor is
//     then inverted in place, so M^{-1} = L^{-T} L^{-1} is applied by two
//     block-wide matrix-vector products.
//  4. FP64 iterative refinement: r = h - (G + lambda I) beta with G beta
//     recomputed from the rows in FP64 each pass (one warp per row, phi
//     formed once per row for both products), delta = M^{-1} r, until the
//     estimated remaining error (step * rho / (1 - rho), rho the step ratio)
//     is below 1e-13 of beta.  Systems that fail the FP32 factorisation,
//     stall, or carry bad inputs are appended to the FP64 resolve list.
// One operand stage (hi, lo) and two row stages keep a CTA near 110 KB of
// shared memory, so two CTAs share an SM and one's solve phase overlaps the
// other's tensor-core loop.
// Every wait on an mbarrier is bounded; TMEM is allocated once per CTA and
// always released before the CTA exits.
#include <algorithm>

#include "ridge.cuh"
#include "tcgen05.cuh"

namespace art {
namespace {

constexpr int kTcThreads = 256;
constexpr int kKC = 32;                    // data rows per stage (MMA K per stage)
constexpr int kPmax = 160;
constexpr int kGroups = kPmax / 8;         // 8-feature core-matrix groups
constexpr int kKE = 4;                     // TF32 elements per 16-byte core-matrix row
constexpr int kKM = 8;                     // MMA K of kind::tf32
constexpr int kLBO = 128;                  // bytes between K-adjacent core matrices
constexpr int kSBO = (kKC / kKE) * 128;    // bytes between 8-feature groups
constexpr int kOpBytes = kGroups * kSBO;   // one operand array (hi or lo)
constexpr int kMaxRefine = 14;
constexpr int kRefRows = 3;                // rows per warp step in the refinement passes
constexpr int kGenRows = kKC / (kTcThreads / 32);  // operand rows generated per warp and chunk
constexpr int kLaneFeat = kPmax / 32;      // features per lane
static_assert(kGenRows == 4, "a warp's rows form one K-row of core matrices");
// TMEM accumulation chains are restarted every kDrainChunks stages: the
// FP32 accumulator of the tensor core loses low bits on every step, so the
// chain length bounds the Gram error (~steps * 2^-24 relative); drained
// partial Grams are summed in shared memory with round-to-nearest adds.
constexpr int kDrainChunks = 4;

// Shared-memory matrix descriptor: K-major, no swizzle (layout type 0),
// LBO = K-direction core-matrix stride, SBO = 8-row group stride, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) { return smem_desc_kmajor(addr, kLBO, kSBO); }
// ------------------------------------------------------------- smem layout
struct TcLayout {
  size_t x[2], y[2], w[2], op, bars, tmem, gram, vec, fidx, total;
};
__host__ __device__ inline size_t a16(size_t v) { return (v + 15) & ~(size_t)15; }
__host__ __device__ inline TcLayout tc_layout(int pmax, int dmax, int factor_bytes) {
  TcLayout L;
  size_t o = 0;
  for (int s = 0; s < 2; ++s) {
    L.x[s] = o; o = a16(o + (size_t)kKC * dmax * 8 + 16);
    L.y[s] = o; o = a16(o + (size_t)kKC * 8 + 16);
    L.w[s] = o; o = a16(o + (size_t)kKC * 8 + 16);
  }
  o = (o + 127) & ~(size_t)127;
  L.op = o; o = a16(o + (size_t)2 * kOpBytes);     // one stage: hi, lo
  L.bars = o; o = a16(o + 4 * 8);
  L.tmem = o; o = a16(o + 16);
  L.gram = o; o = a16(o + (size_t)pmax * (pmax + 1) / 2 * factor_bytes);
  L.vec = o; o = a16(o + (size_t)7 * (pmax + 1) * 8);
  L.fidx = o; o = a16(o + (size_t)kPmax * 4);
  L.total = o;
  return L;
}


struct TcState {
  uint32_t load_issued[2];
  uint32_t load_uses[2];
  uint32_t mma_commits[2];
  uint32_t mma_waits[2];
};

template <typename TF>
__global__ void __launch_bounds__(kTcThreads, sizeof(TF) == 4 ? 2 : 1) ridge_tc_kernel(RidgeArgs a, RidgeLists L,
                                                                 uint32_t tmem_cols) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_item, s_fail, s_flag;
  __shared__ double s_scalar[8];
  const TcLayout lay = tc_layout(a.pmax, a.dmax, (int)sizeof(TF));
  uint64_t* load_bar = (uint64_t*)(smem + lay.bars);
  uint64_t* mma_bar = load_bar + 2;
  uint32_t* s_tmem = (uint32_t*)(smem + lay.tmem);
  TF* Gf = (TF*)(smem + lay.gram);
  double* vec = (double*)(smem + lay.vec);
  int16_t* fidx = (int16_t*)(smem + lay.fidx);
  unsigned char* op = smem + lay.op;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  if (warp == 0) {
    tmem_alloc(s_tmem, tmem_cols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int i = 0; i < 4; ++i) mbar_init(&load_bar[i], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  TcState S = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  bool abort = false;
  const int count = L.count[CLS_TENSOR];

  for (;;) {
    if (tid == 0) s_item = atomicAdd(&L.cursor[CLS_TENSOR], 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= count) break;
    const int k = L.list[(int64_t)CLS_TENSOR * a.K + item];
    const RidgeItem it = load_item(a, k);
    const int p = it.p, d = it.d;
    const int P16 = (p + 15) & ~15;
    const bool two = P16 > 128;
    const int N1 = P16, N2 = two ? P16 - 128 : 0;
    const int g0 = two ? (P16 - 128) / 8 : 0;
    const int64_t nchunks = (it.n + kKC - 1) / kKC;
    if (nchunks == 0) {  // nothing to accumulate: the FP64 form reports the status
      if (tid == 0) push_list(L, a.K, CLS_RESOLVE, k);
      continue;
    }
    for (int f = tid; f < P16; f += kTcThreads) {
      int fa_ = -3, fb_ = -1;
      if (f < p) feature_factors(d, it.kind, f, fa_, fb_);
      fidx[2 * f] = (int16_t)fa_;
      fidx[2 * f + 1] = (int16_t)fb_;
    }
    // exact h and diag partial sums of this lane's features over its warp's rows
    double hacc[kLaneFeat], dacc[kLaneFeat];
#pragma unroll
    for (int m = 0; m < kLaneFeat; ++m) hacc[m] = dacc[m] = 0.0;
    int bad = 0;
    if (tid == 0) {
      for (int64_t c = 0; c < min((int64_t)2, nchunks); ++c) {
        const int64_t rr = c * kKC;
        const int rows = (int)min((int64_t)kKC, it.n - rr);
        Granules gx = granules(a.x + it.xoff + rr * d, (uint64_t)rows * d * 8);
        Granules gy = granules(a.y + it.r0 + rr, (uint64_t)rows * 8);
        Granules gw = a.w ? granules(a.w + it.r0 + rr, (uint64_t)rows * 8) : Granules{nullptr, 0, 0};
        mbar_arrive_expect_tx(&load_bar[c], gx.bytes + gy.bytes + gw.bytes);
        bulk_g2s(smem + lay.x[c], gx.base, gx.bytes, &load_bar[c]);
        bulk_g2s(smem + lay.y[c], gy.base, gy.bytes, &load_bar[c]);
        if (a.w) bulk_g2s(smem + lay.w[c], gw.base, gw.bytes, &load_bar[c]);
      }
    }
    for (int64_t c = 0; c < min((int64_t)2, nchunks); ++c) S.load_issued[c]++;
    __syncthreads();
    // this lane's feature factors, packed as (a + 8) | (b + 8) << 8
    int gfab[kLaneFeat];
#pragma unroll
    for (int m = 0; m < kLaneFeat; ++m) {
      const int f = lane + 32 * m;
      gfab[m] = f < P16 ? (fidx[2 * f] + 8) | ((fidx[2 * f + 1] + 8) << 8) : 5 | (7 << 8);
    }
    const uint32_t id1 = idesc_tf32(128, N1), id2 = idesc_tf32(128, two ? N2 : 16);
    for (int64_t c = 0; c < nchunks && !abort; ++c) {
      const int st = (int)(c & 1);
      const bool okl = mbar_wait(&load_bar[st], S.load_uses[st] & 1);
      const int rows = (int)min((int64_t)kKC, it.n - c * kKC);
      const double* xs = (const double*)(smem + lay.x[st] +
                                         (((uintptr_t)(a.x + it.xoff + c * kKC * d)) & 15));
      const double* ys = (const double*)(smem + lay.y[st] +
                                         (((uintptr_t)(a.y + it.r0 + c * kKC)) & 15));
      const double* ws = a.w ? (const double*)(smem + lay.w[st] +
                                               (((uintptr_t)(a.w + it.r0 + c * kKC)) & 15))
                             : nullptr;
      // input checks and the per-row q y and sqrt(q) need only this chunk's
      // rows, so they run while the tensor core may still hold the operand
      // buffer (the previous chunk's generation finished reading them)
      if (okl)
        for (int e = tid; e < rows * d; e += kTcThreads) bad |= isfinite(xs[e]) ? 0 : 1;
      // warp w generates rows 4w .. 4w+3 of the chunk (one K-row of core
      // matrices), lane l the features l + 32 m; lanes 0..3 form the per-row
      // sqrt(q) and q y of the warp's rows and broadcast them
      const int rw = kGenRows * warp;
      double sqr[kGenRows], qyr[kGenRows];
      const double* xw[kGenRows];
      {
        double sq_l = 0.0, qy_l = 0.0;
        if (okl && lane < kGenRows && rw + lane < rows) {
          const double yv = ys[rw + lane];
          bad |= isfinite(yv) ? 0 : 1;
          const double wv = ws ? ws[rw + lane] : 1.0;
          if (!(wv >= 0.0) || !isfinite(wv)) bad |= 2;
          const double qv = fmax(wv, a.weight_floor);
          qy_l = qv * yv;
          sq_l = sqrt(qv);
        }
#pragma unroll
        for (int u = 0; u < kGenRows; ++u) {
          sqr[u] = __shfl_sync(0xffffffffu, sq_l, u);
          qyr[u] = __shfl_sync(0xffffffffu, qy_l, u);
          xw[u] = xs + (int64_t)(rw + u < rows ? rw + u : 0) * d;
        }
      }
      // one operand buffer: every MMA issued so far (chunks c-2 on barrier st,
      // c-1 on barrier st^1) must be done before it is rewritten; a drain
      // since then has already consumed those commits
      const bool p0 = S.mma_waits[st] < S.mma_commits[st];
      const bool p1 = S.mma_waits[st ^ 1] < S.mma_commits[st ^ 1];
      bool okm = p0 ? mbar_wait(&mma_bar[st], S.mma_waits[st] & 1) : true;
      okm = okm && (p1 ? mbar_wait(&mma_bar[st ^ 1], S.mma_waits[st ^ 1] & 1) : true);
      if (!__syncthreads_and(okl && okm)) { abort = true; break; }
      S.load_uses[st]++;
      if (p0) S.mma_waits[st]++;
      if (p1) S.mma_waits[st ^ 1]++;
      unsigned char* hi = op;
      unsigned char* lo = hi + kOpBytes;
#pragma unroll
      for (int m = 0; m < kLaneFeat; ++m) {
        const int f = lane + 32 * m;
        if (f < P16) {
          const int ia = (gfab[m] & 255) - 8, ib = (gfab[m] >> 8) - 8;
          uint32_t ph[kGenRows], pl[kGenRows];
#pragma unroll
          for (int u = 0; u < kGenRows; ++u) {
            float v = 0.0f;
            if (rw + u < rows && ia != -3) {
              const double phi = (ia < 0 ? 1.0 : xw[u][ia]) * (ib < 0 ? 1.0 : xw[u][ib]);
              // h += phi (q y) and diag += (sqrt(q) phi)^2: one product fewer
              // and no separate y load per feature
              const double sphi = sqr[u] * phi;
              hacc[m] = fma(phi, qyr[u], hacc[m]);
              dacc[m] = fma(sphi, sphi, dacc[m]);
              v = (float)sphi;
            }
            ph[u] = to_tf32(v);
            pl[u] = to_tf32(v - __uint_as_float(ph[u]));
          }
          const size_t off = (size_t)(f >> 3) * kSBO + (size_t)warp * 128 + (size_t)(f & 7) * 16;
          *(uint4*)(hi + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *(uint4*)(lo + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
      }
      fence_proxy_async();  // operand writes -> visible to the tensor core
      __syncthreads();
      if (c + 2 < nchunks) S.load_issued[st]++;
      if (tid == 0) {
        if (c + 2 < nchunks) {
          const int64_t rr = (c + 2) * kKC;
          const int r2 = (int)min((int64_t)kKC, it.n - rr);
          Granules gx = granules(a.x + it.xoff + rr * d, (uint64_t)r2 * d * 8);
          Granules gy = granules(a.y + it.r0 + rr, (uint64_t)r2 * 8);
          Granules gw = a.w ? granules(a.w + it.r0 + rr, (uint64_t)r2 * 8) : Granules{nullptr, 0, 0};
          mbar_arrive_expect_tx(&load_bar[st], gx.bytes + gy.bytes + gw.bytes);
          bulk_g2s(smem + lay.x[st], gx.base, gx.bytes, &load_bar[st]);
          bulk_g2s(smem + lay.y[st], gy.base, gy.bytes, &load_bar[st]);
          if (a.w) bulk_g2s(smem + lay.w[st], gw.base, gw.bytes, &load_bar[st]);
        }
        tc_fence_after();
        const uint32_t hb = smem_u32(hi), lb = smem_u32(lo);
#pragma unroll
        for (int s = 0; s < kKC / kKM; ++s) {
          const uint32_t ko = (uint32_t)s * (kKM / kKE) * kLBO;
#pragma unroll
          for (int prod = 0; prod < 3; ++prod) {
            const uint32_t A = (prod == 2) ? lb : hb;
            const uint32_t B = (prod == 1) ? lb : hb;
            const uint32_t acc = ((c % kDrainChunks) == 0 && s == 0 && prod == 0) ? 0u : 1u;
            mma_tf32(tmem, smem_desc(A + ko), smem_desc(B + ko), id1, acc);
            if (two)
              mma_tf32(tmem + (uint32_t)N1, smem_desc(A + (uint32_t)g0 * kSBO + ko),
                       smem_desc(B + 16u * kSBO + ko), id2, acc);
          }
        }
        mma_commit(&mma_bar[st]);
      }
      S.mma_commits[st]++;
      const bool seg_end = ((c + 1) % kDrainChunks) == 0 || c + 1 == nchunks;
      if (seg_end) {
        // wait for every MMA of this segment, then add the partial Gram from TMEM
        bool okw = true;
        for (int s2 = 0; s2 < 2 && okw; ++s2)
          while (S.mma_waits[s2] < S.mma_commits[s2]) {
            if (!mbar_wait(&mma_bar[s2], S.mma_waits[s2] & 1)) { okw = false; break; }
            S.mma_waits[s2]++;
          }
        if (!__syncthreads_and(okw)) { abort = true; break; }
        tc_fence_after();
        const bool first = c < kDrainChunks;
        const int sp = warp & 3, half = warp >> 2;
        const int row = 32 * sp + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * sp) << 16);
        for (int cb = half * 16; cb < N1; cb += 32) {
          float v[16];
          tmem_ld16(lane_base + (uint32_t)cb, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = cb + j;
            // lower entries of tile 1, plus its upper block G[row < 128][col >= 128],
            // which is the transpose of the lower-left block of features >= 128
            if (row < p && col < p && (col <= row || col >= 128)) {
              TF* gp = (col <= row) ? &Gf[pk(row, col)] : &Gf[pk(col, row)];
              *gp = first ? (TF)v[j] : *gp + (TF)v[j];
            }
          }
        }
        if (two) {
          const int frow = g0 * 8 + row;
          for (int cb = half * 16; cb < N2; cb += 32) {
            float v[16];
            tmem_ld16(lane_base + (uint32_t)(N1 + cb), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int col = 128 + cb + j;
              if (frow >= 128 && frow < p && col <= frow) {
                TF* gp = &Gf[pk(frow, col)];
                *gp = first ? (TF)v[j] : *gp + (TF)v[j];
              }
            }
          }
        }
        tc_fence_before();
        __syncthreads();
      }
    }
    if (abort || !__syncthreads_and(!abort)) {
      if (tid == 0) { atomicExch(L.err, 1); a.status[k] = -5; }
      abort = true;
      break;
    }
    tc_fence_before();
    if (a.gram_out) {  // Gram-only call: dump the tensor-core Gram and move on
      __syncthreads();
      const int E = p * (p + 1) / 2;
      for (int e = tid; e < E; e += kTcThreads) a.gram_out[(int64_t)k * a.gram_stride + e] = (float)Gf[e];
      if (tid == 0) a.status[k] = 0;
      __syncthreads();
      continue;
    }
    // ---- reduce exact h and diag over the warps (fixed order)
    double* red = (double*)op;  // operand buffers are idle now: [warp][P16] pairs
#pragma unroll
    for (int m = 0; m < kLaneFeat; ++m) {
      const int f = lane + 32 * m;
      if (f < P16) {
        red[2 * (warp * P16 + f)] = hacc[m];
        red[2 * (warp * P16 + f) + 1] = dacc[m];
      }
    }
    {
      const int bw = __syncthreads_or(bad & 2), bx = __syncthreads_or(bad & 1);
      bad = (bw ? 2 : 0) | (bx ? 1 : 0);
    }
    const int vs = a.pmax + 1;  // vector stride (tc_layout reserves 7 * vs)
    double* h = vec;
    double* dg = vec + vs;
    double* beta = vec + 2 * vs;
    double* r = vec + 3 * vs;
    double* v1 = vec + 4 * vs;
    double* v2 = vec + 5 * vs;
    for (int f = tid; f < p; f += kTcThreads) {
      double hs = 0.0, ds = 0.0;
      for (int wv = 0; wv < kTcThreads / 32; ++wv) {
        hs += red[2 * (wv * P16 + f)];
        ds += red[2 * (wv * P16 + f) + 1];
      }
      h[f] = hs;
      dg[f] = ds;
    }
    __syncthreads();
    if (tid == 0) {
      double tr = 0.0;
      for (int f = 0; f < p; ++f) tr += dg[f];
      const double lam = it.ridge * tr / p;
      s_scalar[0] = lam;
      L.lambda[k] = lam;
    }
    __syncthreads();
    const double lam = s_scalar[0];
    if (bad) {
      if (tid == 0) push_list(L, a.K, CLS_RESOLVE, k);
      continue;
    }
    for (int f = tid; f < p; f += kTcThreads) Gf[pk(f, f)] = (TF)(dg[f] + lam);
    __syncthreads();
    const bool want_cond = (a.cond != nullptr) || (a.solver == ART_SOLVER_AUTO);
    if (want_cond && warp == 0) {
      const double an = warp_sym_norm1(Gf, p);
      if (lane == 0) s_scalar[1] = an;
    }
    const int fail = chol_packed32<TF>(Gf, p, &s_fail);
    if (fail) {
      if (tid == 0) push_list(L, a.K, CLS_RESOLVE, k);
      continue;
    }
    double cond = __longlong_as_double(0x7ff8000000000000ll);
    if (want_cond) {  // 1-norm estimate from the factor (dpocon's method)
      if (warp == 0) {
        const double est = warp_inv_norm1_estimate<TF>(Gf, p, v1, v2);
        if (lane == 0) {
          const double an = s_scalar[1];
          s_scalar[2] = (est > 0.0 && isfinite(est) && an > 0.0) ? 1.0 / (an * est) : 0.0;
        }
      }
      __syncthreads();
      const double rcond = s_scalar[2];
      if (a.solver == ART_SOLVER_AUTO && rcond < a.rcond_threshold) {
        // let the FP64 form apply the auto policy exactly
        if (tid == 0) push_list(L, a.K, CLS_RESOLVE, k);
        continue;
      }
      cond = rcond > 0.0 ? sqrt(1.0 / fmin(rcond, 1.0)) : __longlong_as_double(0x7ff0000000000000ll);
    }
    // ---- M^{-1} = L^{-T} L^{-1}: invert the factor in place (the operand
    // buffers are idle and hold the panel scratch), then every application
    // is two block-wide triangular matrix-vector products.
    tri_inv_packed32<TF>(Gf, p, (TF*)op);
    double* tvec = vec + 6 * vs;
    auto apply_minv = [&](const double* v, double* out) { apply_inv_factor<TF>(Gf, p, v, tvec, out); };
    double* part = (double*)op;  // [8 row slots][kPmax], after the row passes
    // refinement row stages also live in the operand buffers: two stages of
    // RC rows of x (and w), RC a multiple of 8 (one row per warp per step)
    int RC = (int)(((size_t)kOpBytes - 128) / ((size_t)a.dmax * 8 + 8)) & ~7;
    RC = RC > 256 ? 256 : RC;
    const size_t rx_bytes = a16((size_t)RC * a.dmax * 8 + 32);
    const size_t rstage = rx_bytes + a16((size_t)RC * 8 + 32);
    auto issue_rows = [&](int64_t c, int st) {
      const int64_t rr = c * RC;
      const int rows = (int)min((int64_t)RC, it.n - rr);
      Granules gx = granules(a.x + it.xoff + rr * it.d, (uint64_t)rows * it.d * 8);
      Granules gw = a.w ? granules(a.w + it.r0 + rr, (uint64_t)rows * 8) : Granules{nullptr, 0, 0};
      mbar_arrive_expect_tx(&load_bar[st], gx.bytes + gw.bytes);
      bulk_g2s(op + st * rstage, gx.base, gx.bytes, &load_bar[st]);
      if (a.w) bulk_g2s(op + st * rstage + rx_bytes, gw.base, gw.bytes, &load_bar[st]);
    };
    // ---- FP64 iterative refinement.  Residual passes: one warp per row (8
    // rows per step), lane l owns features l + 32 m (m < 5) with their beta
    // in registers; phi is formed once per row and used for both
    // e_k = q_k phi_k . beta (warp shuffle sum) and the accumulation of
    // e_k phi_k; the 8 row slots are summed in a fixed order at the end.
    const int slot = warp, fl = lane;
    int rfa[5], rfb[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const int f = fl + 32 * m;
      rfa[m] = f < p ? fidx[2 * f] : -3;
      rfb[m] = f < p ? fidx[2 * f + 1] : -1;
    }
    apply_minv(h, beta);   // beta_0 = M^{-1} h
    double nd_prev = 0.0;
    {
      if (warp == 0) {
        double m0 = 0.0;
        for (int f = lane; f < p; f += 32) m0 = fmax(m0, fabs(beta[f]));
        m0 = warp_max(m0);
        if (lane == 0) s_scalar[3] = m0;
      }
      __syncthreads();
      nd_prev = s_scalar[3];
    }
    int outcome = (nd_prev <= 1e300) ? 0 : 2;  // 1 converged, 2 stalled/failed
    uint32_t info = 0;
    int passes = 0;
    for (int iter = 1; iter < kMaxRefine && outcome == 0; ++iter) {
      passes = iter;
      double bt[5], accb[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const int f = fl + 32 * m;
        bt[m] = f < p ? beta[f] : 0.0;
        accb[m] = 0.0;
      }
      // rows stream through the two row stages again (bulk copies of x and
      // w, prefetched two chunks ahead); warp `slot` takes rows slot, slot+8,
      // ... of each chunk, so every warp stays converged
      const int64_t nch = (it.n + RC - 1) / RC;
      if (tid == 0)
        for (int64_t c = 0; c < min((int64_t)2, nch); ++c) issue_rows(c, (int)c);
      for (int64_t c = 0; c < min((int64_t)2, nch); ++c) S.load_issued[c]++;
      for (int64_t c = 0; c < nch && !abort; ++c) {
        const int st = (int)(c & 1);
        const bool okl = mbar_wait(&load_bar[st], S.load_uses[st] & 1);
        if (!__syncthreads_and(okl)) { abort = true; break; }
        S.load_uses[st]++;
        const int rows = (int)min((int64_t)RC, it.n - c * RC);
        const double* xs = (const double*)(op + st * rstage +
                                           (((uintptr_t)(a.x + it.xoff + c * RC * d)) & 15));
        const double* ws = a.w ? (const double*)(op + st * rstage + rx_bytes +
                                                 (((uintptr_t)(a.w + it.r0 + c * RC)) & 15))
                               : nullptr;
        // kRefRows rows per warp and step, their dot products and shuffle
        // sums interleaved; the accumulation still runs row by row in the
        // warp's row order (the tail test is warp-uniform)
        constexpr int kStep = kTcThreads / 32;
        for (int j = slot; j < rows; j += kStep * kRefRows) {
          double ph[kRefRows][5], dot[kRefRows];
#pragma unroll
          for (int u = 0; u < kRefRows; ++u) {
            const int jj = j + kStep * u;
            dot[u] = 0.0;
            const double* xk = xs + (jj < rows ? jj : j) * d;
#pragma unroll
            for (int m = 0; m < 5; ++m) {
              const int ua = rfa[m], ub = rfb[m];
              const double va = ua >= 0 ? xk[ua] : (ua == -1 ? 1.0 : 0.0);
              const double vb = ub >= 0 ? xk[ub] : 1.0;
              ph[u][m] = va * vb;
              dot[u] = fma(ph[u][m], bt[m], dot[u]);
            }
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int u = 0; u < kRefRows; ++u) dot[u] += __shfl_xor_sync(0xffffffffu, dot[u], o);
#pragma unroll
          for (int u = 0; u < kRefRows; ++u) {
            const int jj = j + kStep * u;
            if (jj < rows) {
              const double e = fmax(ws ? ws[jj] : 1.0, a.weight_floor) * dot[u];
#pragma unroll
              for (int m = 0; m < 5; ++m) accb[m] = fma(e, ph[u][m], accb[m]);
            }
          }
        }
        __syncthreads();  // every warp is done with this stage
        if (c + 2 < nch) {
          if (tid == 0) issue_rows(c + 2, st);
          S.load_issued[st]++;
        }
      }
      if (abort) break;
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const int f = fl + 32 * m;
        if (f < p) part[slot * kPmax + f] = accb[m];
      }
      __syncthreads();
      for (int f = tid; f < p; f += kTcThreads) {
        double sacc = 0.0;
        for (int sl = 0; sl < kTcThreads / 32; ++sl) sacc += part[sl * kPmax + f];
        r[f] = h[f] - lam * beta[f] - sacc;
      }
      __syncthreads();
      apply_minv(r, v1);   // correction
      if (warp == 0) {
        double nd = 0.0, nb = 0.0;
        for (int f = lane; f < p; f += 32) {
          const double b = beta[f] + v1[f];
          beta[f] = b;
          nd = fmax(nd, fabs(v1[f]));
          nb = fmax(nb, fabs(b));
        }
        nd = warp_max(nd);
        nb = warp_max(nb);
        if (lane == 0) {
          int out = 0;
          const double rho = nd_prev > 0.0 ? nd / nd_prev : 0.0;
          if (!(nd <= 1e300) || !(nb <= 1e300)) out = 2;                       // non-finite
          else if (nd <= 2.3e-16 * nb) out = 1;                                 // at working precision
          else if (rho < 0.75 && nd * rho / (1.0 - rho) <= 1e-13 * nb) out = 1; // remaining error tiny
          else if (rho >= 0.75) out = (nd <= 1e-12 * nb) ? 1 : 2;              // stalled
          else if (iter == kMaxRefine - 1) out = (nd <= 1e-12 * nb) ? 3 : 2;
          s_flag = out;
          s_scalar[3] = nd;
        }
      }
      __syncthreads();
      outcome = s_flag;
      nd_prev = s_scalar[3];
      if (outcome == 3) { outcome = 1; info |= ART_INFO_REFINE_CAP; }
    }
    if (abort) {  // a bounded wait gave up in a refinement pass
      if (tid == 0) { atomicExch(L.err, 1); a.status[k] = -5; }
      break;
    }
    info |= (uint32_t)min(passes, 255) << ART_INFO_REFINE_SHIFT;
    if (outcome != 1) {
      if (tid == 0) {
        push_list(L, a.K, CLS_RESOLVE, k);
        if (a.info) a.info[k] = info;  // the FP64 form ORs its own bits in
      }
      continue;
    }
    for (int f = tid; f < p; f += kTcThreads) a.beta[(int64_t)k * a.beta_stride + f] = beta[f];
    if (tid == 0) {
      a.status[k] = 0;
      if (a.ridge_eff) a.ridge_eff[k] = lam;
      if (a.cond) a.cond[k] = cond;
      if (a.info) a.info[k] = info;
    }
    __syncthreads();
  }
  // release TMEM after bounded waits for this CTA's MMAs and bulk copies in flight
  for (int st = 0; st < 2; ++st) {
    while (S.mma_waits[st] < S.mma_commits[st]) {
      if (!mbar_wait(&mma_bar[st], S.mma_waits[st] & 1)) break;
      S.mma_waits[st]++;
    }
    while (S.load_uses[st] < S.load_issued[st]) {
      if (!mbar_wait(&load_bar[st], S.load_uses[st] & 1)) break;
      S.load_uses[st]++;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, tmem_cols);
}

template <typename TF>
int launch_tc(const RidgeArgs& a, const RidgeLists& L, cudaStream_t s, const char* name) {
  auto kern = ridge_tc_kernel<TF>;
  const int P16 = (std::min(a.pmax, kPmax) + 15) & ~15;
  const int cols_needed = P16 + (P16 > 128 ? P16 - 128 : 0);
  uint32_t cols = 32;
  while ((int)cols < cols_needed) cols <<= 1;
  size_t smem = tc_layout(a.pmax, a.dmax, (int)sizeof(TF)).total;
  // TMEM: CTAs resident on one SM must fit 512 columns together; widen the
  // shared-memory request if occupancy would allow more CTAs than that.
  const int max_ctas = (int)(512 / cols);
  int occ = 0;
  for (;;) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
      cudaGetLastError();
      set_error("%s: cannot reserve %zu bytes of shared memory", name, smem);
      return ART_E_UNSUPPORTED;
    }
    occ = resident_ctas((const void*)kern, kTcThreads, smem);
    if (occ <= max_ctas || smem + 8 * 1024 > 200 * 1024) break;
    smem += 8 * 1024;
  }
  if (occ > max_ctas) {
    set_error("%s: cannot place CTAs within TMEM capacity (occ %d, cols %u)", name, occ, cols);
    return ART_E_UNSUPPORTED;
  }
  const int64_t grid = std::min<int64_t>((int64_t)device_sm_count() * occ, a.K);
  prof_begin(name, s);
  kern<<<(unsigned)std::max<int64_t>(grid, 1), kTcThreads, smem, s>>>(a, L, cols);
  prof_end(s);
  count_launch();
  return check_launch(name);
}

}  // namespace

int launch_ridge_tensor(const RidgeArgs& a, const RidgeLists& L, cudaStream_t s) {
  if (a.dmax > ART_MAX_DIM) {
    set_error("mixed precision requires max_dim <= %d", ART_MAX_DIM);
    return ART_E_UNSUPPORTED;
  }
  if ((a.options & ART_RIDGE_OPT_FP64_FACTOR) && !a.gram_out)
    return launch_tc<double>(a, L, s, "ridge_tc<f64 factor>");
  return launch_tc<float>(a, L, s, "ridge_tc");
}

}  // namespace art
