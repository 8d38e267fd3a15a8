// har.cu -- hit-and-run chains in node polytopes {lo <= x <= hi, A x <= b}.
//
// Follows the reference transitions:
//  * ART_HAR_BATCHED: sample_precomputed_chains(_parallel)
//    (art/_numba_sampling.py:9-167): Gaussian directions used unnormalised,
//    slacks s = b - A x updated incrementally (s -= t * A u), chord bounds
//    from the signs of A u (exact zero tests), t = t_lo + U (t_hi - t_lo),
//    a sample after every `thinning` steps following `burn_in`.
//  * ART_HAR_SCALAR: HitAndRunSampler.sample (art/sampling.py:445-495,
//    _step_interval 540-564): unit directions, slack recomputed from x each
//    step, |A u| > 1e-14 tests, samples at steps burn_in + k*thinning.
//
// Layout: a team of L lanes (L = next power of two >= ceil(d/2), L <= 32)
// advances one chain; lane l owns coordinates 2l and 2l+1, so one Philox
// block gives both of its normals.  Box rows (+e_i, -e_i) are applied
// structurally: A u = +-u_i exactly, as in the reference's dense matmul.
// Oblique rows are held in shared memory and reduced across the team.
#include <algorithm>
#include "common.cuh"

namespace art {
namespace {

constexpr int kHarThreads = 256;
constexpr double kScalarParallelTol = 1e-14;  // sampling.py:552-553
constexpr double kFeasTol = 1e-10;             // sampling.py:438, domain.py:40

struct HarArgs {
  int64_t n_poly;
  int d;
  const double* lo;
  const double* hi;
  const int64_t* row_offsets;
  const double* A;
  const double* b;
  const double* maps;  // [n_poly][d][d] or NULL
  int64_t n_chains;
  const int32_t* polytope;
  double* x;
  const uint64_t* seeds;
  const double* dirs;
  const double* unif;
  int mode;
  int burn_in, thinning, n_rounds;
  uint64_t counter_base;
  double* samples;
  int32_t* status;
};

template <int L>
__device__ __forceinline__ double team_sum(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int L>
__device__ __forceinline__ double team_max(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <int L>
__device__ __forceinline__ double team_min(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <int L>
__device__ __forceinline__ int team_or(int v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Oblique rows of a team's polytope live in shared memory (team stride
// MAXK * d + 1 doubles, odd, so the teams of a warp use different banks);
// row r's slack, bound and direction product are kept by lane r % L only.
template <int L, int MAXK>
__host__ __device__ constexpr size_t har_team_stride(int d) { return (size_t)MAXK * d + 1; }

// Teams of 4 or more lanes on polytopes of up to 16 rows are held to two
// resident CTAs per SM (128 registers a thread); narrower teams and longer
// row lists take the registers they need.
constexpr int har_min_ctas(int L, int MAXK) { return (L >= 4 && MAXK <= 16) ? 2 : 1; }

template <int L, int MAXK>
__global__ void __launch_bounds__(kHarThreads, har_min_ctas(L, MAXK)) har_kernel(HarArgs a) {
  extern __shared__ double s_rows[];
  constexpr int OWN = (MAXK + L - 1) / L;  // rows owned by each lane
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t chain_raw = gt / L;
  const int lane = (int)(gt % L);
  // Teams past the end keep running (masked) so that full-warp shuffles stay valid.
  const bool live = chain_raw < a.n_chains;
  const int64_t chain = live ? chain_raw : (a.n_chains - 1);
  const int d = a.d;
  const int i0 = 2 * lane, i1 = 2 * lane + 1;
  const bool h0 = i0 < d, h1 = i1 < d;
  const int pj = a.polytope[chain];
  const int64_t rb = a.row_offsets[pj];
  const int k = (int)(a.row_offsets[pj + 1] - rb);
  const bool scalar = a.mode == ART_HAR_SCALAR;
  int status = 0;
  if (k > MAXK) status = 3;
  double x0 = h0 ? a.x[chain * d + i0] : 0.0;
  double x1 = h1 ? a.x[chain * d + i1] : 0.0;
  const bool box = a.lo != nullptr;
  double lo0 = 0, lo1 = 0, hi0 = 0, hi1 = 0;
  if (box) {
    lo0 = h0 ? a.lo[(int64_t)pj * d + i0] : 0.0;
    lo1 = h1 ? a.lo[(int64_t)pj * d + i1] : 0.0;
    hi0 = h0 ? a.hi[(int64_t)pj * d + i0] : 0.0;
    hi1 = h1 ? a.hi[(int64_t)pj * d + i1] : 0.0;
  }
  double* Ar = s_rows + (size_t)(threadIdx.x / L) * har_team_stride<L, MAXK>(d);
  for (int e = lane; e < MAXK * d; e += L) {
    const int r = e / d, i = e - r * d;
    Ar[e] = (r < k && status == 0) ? a.A[(rb + r) * d + i] : 0.0;
  }
  __syncwarp();
  // this lane's coefficient of row r on its two coordinates
  auto arow = [&](int r, double v0, double v1) {
    return (h0 ? Ar[r * d + i0] * v0 : 0.0) + (h1 ? Ar[r * d + i1] * v1 : 0.0);
  };
  double br[OWN], so[OWN], au[OWN];
#pragma unroll
  for (int m = 0; m < OWN; ++m) {
    const int r = m * L + lane;
    br[m] = (r < MAXK && r < k && status == 0) ? a.b[rb + r] : 0.0;
    so[m] = 0.0;
    au[m] = 0.0;
  }
  // initial slacks s = b - A x (numba path: sampling.py:648)
  double shi0 = hi0 - x0, shi1 = hi1 - x1, slo0 = x0 - lo0, slo1 = x1 - lo1;
  int bad_start = 0;
  if (box) {
    if (h0 && (shi0 < -kFeasTol || slo0 < -kFeasTol)) bad_start = 1;
    if (h1 && (shi1 < -kFeasTol || slo1 < -kFeasTol)) bad_start = 1;
  }
#pragma unroll
  for (int r = 0; r < MAXK; ++r) {
    const double ax = team_sum<L>(arow(r, x0, x1));
    if (r % L == lane) {
      so[r / L] = br[r / L] - ax;
      if (r < k && so[r / L] < -kFeasTol) bad_start = 1;
    }
  }
  bad_start = team_or<L>(bad_start);
  const int kwarp = __reduce_max_sync(0xffffffffu, status == 0 ? k : 0);
  if (bad_start && status == 0) status = 2;
  const uint32_t key0 = a.seeds ? (uint32_t)a.seeds[chain] : 0u;
  const uint32_t key1 = a.seeds ? (uint32_t)(a.seeds[chain] >> 32) : 0u;
  const int total = a.burn_in + a.n_rounds * a.thinning;
  const int64_t C = a.n_chains;
  int64_t ucur = 0;  // uniform cursor (scalar mode skips draws on zero directions)
  // next step that keeps a sample and its index: scalar mode keeps steps
  // burn_in + j * thinning (none on a zero direction), batched mode the last
  // step of each thinning block after burn_in
  int keep_step = scalar ? a.burn_in : a.burn_in + a.thinning - 1;
  int keep_idx = 0;
  // one step per iteration: the body is long, and unrolling it only grows the
  // code the warps fetch
#pragma unroll 1
  for (int step = 0; step < total; ++step) {
    double u0, u1;
    if (a.dirs) {
      const double* dp = a.dirs + (chain * total + step) * (int64_t)d;
      u0 = h0 ? dp[i0] : 0.0;
      u1 = h1 ? dp[i1] : 0.0;
    } else {
      const uint64_t ctr = a.counter_base + (uint64_t)step;
      Philox4 r = philox4x32_10((uint32_t)ctr, (uint32_t)(ctr >> 32), (uint32_t)lane, 0u, key0,
                                key1);
      normal_pair_f32(r, u0, u1);
      if (!h0) u0 = 0.0;
      if (!h1) u1 = 0.0;
      if (a.maps) {  // covariance-shaped direction u = M z, z gathered across the team
        const double* M = a.maps + (int64_t)pj * d * d;
        double m0 = 0.0, m1 = 0.0;
        for (int j = 0; j < d; ++j) {
          const double za = __shfl_sync(0xffffffffu, u0, j >> 1, L);
          const double zb = __shfl_sync(0xffffffffu, u1, j >> 1, L);
          const double zj = (j & 1) ? zb : za;
          if (h0) m0 = fma(M[(int64_t)i0 * d + j], zj, m0);
          if (h1) m1 = fma(M[(int64_t)i1 * d + j], zj, m1);
        }
        u0 = m0;
        u1 = m1;
      }
    }
    bool skip = false;
    if (scalar) {
      const double nrm2 = team_sum<L>(u0 * u0 + u1 * u1);
      const double nrm = sqrt(nrm2);
      if (nrm == 0.0) skip = true;
      else { u0 = u0 / nrm; u1 = u1 / nrm; }
      // recompute slacks from x (sampling.py:548-550)
      shi0 = hi0 - x0; shi1 = hi1 - x1; slo0 = x0 - lo0; slo1 = x1 - lo1;
#pragma unroll
      for (int r = 0; r < MAXK; ++r) {
        const double ax = team_sum<L>(arow(r, x0, x1));
        if (r % L == lane) so[r / L] = br[r / L] - ax;
      }
    }
    // rows past the largest count in the warp are zero: skip them (a
    // warp-uniform bound, so the team shuffles stay converged)
#pragma unroll
    for (int r = 0; r < MAXK; ++r) {
      if (r >= kwarp) break;
      const double v = team_sum<L>(arow(r, u0, u1));
      if (r % L == lane) au[r / L] = v;
    }
    if (!skip) {
      const double pos_t = scalar ? kScalarParallelTol : 0.0;
      double tlo = -INFINITY, thi = INFINITY;
      int infeasible = 0;
      auto box_row = [&](double slack, double prod) {
        if (prod > pos_t) thi = fmin(thi, slack / prod);
        else if (prod < -pos_t) tlo = fmax(tlo, slack / prod);
        else if (scalar && slack < -kFeasTol) infeasible = 1;
      };
      if (box) {
        if (h0) { box_row(shi0, u0); box_row(slo0, -u0); }
        if (h1) { box_row(shi1, u1); box_row(slo1, -u1); }
      }
      // each lane walks only the rows it owns (r = m L + lane); min and max
      // do not depend on the order
#pragma unroll
      for (int m = 0; m < OWN; ++m) {
        const int r = m * L + lane;
        if (r < MAXK && r < k) box_row(so[m], au[m]);
      }
      tlo = team_max<L>(tlo);
      thi = team_min<L>(thi);
      infeasible = team_or<L>(infeasible);
      if (status == 0 && (tlo > thi || infeasible)) status = 1;
      double U;
      if (a.unif) {
        U = a.unif[chain * total + (scalar ? ucur : step)];
      } else {
        const uint64_t ctr = a.counter_base + (uint64_t)step;
        Philox4 r = philox4x32_10((uint32_t)ctr, (uint32_t)(ctr >> 32), 0xFFFFFFFFu, 1u, key0,
                                  key1);
        U = u01_closed_open(r.v[0], r.v[1]);
      }
      ++ucur;
      // Separate roundings (no FMA contraction), as numpy/numba evaluate them.
      const double t = __dadd_rn(tlo, __dmul_rn(U, __dsub_rn(thi, tlo)));
      if (status == 0) {
        x0 = __dadd_rn(x0, __dmul_rn(t, u0));
        x1 = __dadd_rn(x1, __dmul_rn(t, u1));
        if (!scalar) {
          shi0 = __dsub_rn(shi0, __dmul_rn(t, u0));
          shi1 = __dsub_rn(shi1, __dmul_rn(t, u1));
          slo0 = __dsub_rn(slo0, __dmul_rn(t, -u0));
          slo1 = __dsub_rn(slo1, __dmul_rn(t, -u1));
#pragma unroll
          for (int m = 0; m < OWN; ++m) so[m] = __dsub_rn(so[m], __dmul_rn(t, au[m]));
        }
      }
    }
    // sample bookkeeping
    int out = -1;
    if (step == keep_step) {
      if (!(scalar && skip)) out = keep_idx;
      ++keep_idx;
      keep_step += a.thinning;
    }
    if (out >= 0 && out < a.n_rounds && live) {
      double* sp = a.samples + ((int64_t)out * C + chain) * d;
      if (h0) sp[i0] = x0;
      if (h1) sp[i1] = x1;
    }
  }
  if (live) {
    if (h0) a.x[chain * d + i0] = x0;
    if (h1) a.x[chain * d + i1] = x1;
    if (lane == 0 && a.status) a.status[chain] = status;
  }
}

template <int L, int MAXK>
int launch_har_k(const HarArgs& a, unsigned grid, cudaStream_t s) {
  const size_t smem = (size_t)(kHarThreads / L) * har_team_stride<L, MAXK>(a.d) * 8;
  if (cudaFuncSetAttribute(har_kernel<L, MAXK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("art_hit_and_run: cannot reserve %zu bytes of shared memory", smem);
    return ART_E_UNSUPPORTED;
  }
  cudaFuncSetAttribute(har_kernel<L, MAXK>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  cudaGetLastError();
  prof_begin("hit_and_run", s);
  har_kernel<L, MAXK><<<grid, kHarThreads, smem, s>>>(a);
  prof_end(s);
  count_launch();
  return check_launch("art_hit_and_run");
}

template <int L>
int launch_har_l(const HarArgs& a, int maxk, cudaStream_t s) {
  const int64_t threads = a.n_chains * L;
  const unsigned grid = (unsigned)((threads + kHarThreads - 1) / kHarThreads);
  if (maxk <= 4) return launch_har_k<L, 4>(a, grid, s);
  if (maxk <= 8) return launch_har_k<L, 8>(a, grid, s);
  if (maxk <= 16) return launch_har_k<L, 16>(a, grid, s);
  return launch_har_k<L, 32>(a, grid, s);
}

}  // namespace
}  // namespace art

using namespace art;

extern "C" int art_hit_and_run(const ArtPolytopes* P, const ArtChains* C, art_stream_t stream) {
  cudaGetLastError();
  if (!P || !C) { set_error("art_hit_and_run: null argument"); return ART_E_INVALID; }
  if (C->count < 0 || P->count < 0) { set_error("art_hit_and_run: negative count"); return ART_E_INVALID; }
  if (C->count == 0) return ART_OK;
  if (P->dim < 1 || P->dim > ART_MAX_DIM) {
    set_error("art_hit_and_run: dim %d outside [1, %d]", P->dim, ART_MAX_DIM);
    return ART_E_UNSUPPORTED;
  }
  if (P->max_rows < 0 || P->max_rows > 32) {
    set_error("art_hit_and_run: max_rows %d outside [0, 32]", P->max_rows);
    return ART_E_UNSUPPORTED;
  }
  if (!P->row_offsets || (P->max_rows > 0 && (!P->A || !P->b)) || ((P->lo == nullptr) != (P->hi == nullptr))) {
    set_error("art_hit_and_run: polytope arrays incomplete");
    return ART_E_INVALID;
  }
  if (!C->polytope || !C->x || (!C->samples && C->n_rounds > 0)) {
    set_error("art_hit_and_run: chain arrays incomplete");
    return ART_E_INVALID;
  }
  if ((C->directions == nullptr) != (C->uniforms == nullptr)) {
    set_error("art_hit_and_run: inject both directions and uniforms, or neither");
    return ART_E_INVALID;
  }
  if (!C->directions && !C->seeds) {
    set_error("art_hit_and_run: seeds are required without injected draws");
    return ART_E_INVALID;
  }
  if (C->mode != ART_HAR_BATCHED && C->mode != ART_HAR_SCALAR) {
    set_error("art_hit_and_run: unknown mode %d", C->mode);
    return ART_E_INVALID;
  }
  if (C->burn_in < 0 || C->thinning < 1 || C->n_rounds < 0) {
    set_error("art_hit_and_run: burn_in >= 0, thinning >= 1, n_rounds >= 0 required");
    return ART_E_INVALID;
  }
  HarArgs a;
  a.n_poly = P->count; a.d = P->dim; a.lo = P->lo; a.hi = P->hi;
  a.maps = P->direction_maps;
  a.row_offsets = P->row_offsets; a.A = P->A; a.b = P->b;
  a.n_chains = C->count; a.polytope = C->polytope; a.x = C->x; a.seeds = C->seeds;
  a.dirs = C->directions; a.unif = C->uniforms; a.mode = C->mode;
  a.burn_in = C->burn_in; a.thinning = C->thinning; a.n_rounds = C->n_rounds;
  a.counter_base = C->counter_base; a.samples = C->samples; a.status = C->status;
  cudaStream_t s = (cudaStream_t)stream;
  const int half = (P->dim + 1) / 2;
  const int maxk = P->max_rows;
  if (half <= 1) return launch_har_l<1>(a, maxk, s);
  if (half <= 2) return launch_har_l<2>(a, maxk, s);
  if (half <= 4) return launch_har_l<4>(a, maxk, s);
  if (half <= 8) return launch_har_l<8>(a, maxk, s);
  if (half <= 16) return launch_har_l<16>(a, maxk, s);
  return launch_har_l<32>(a, maxk, s);
}
