// split.cu -- soft oblique split search for a whole tree level in one launch.
//
// Device form of SoftObliqueSplitter.split (art/splitters.py:252-363) and
// _optimize_from_initialization (365-601) with the objective of
// SoftObliqueRidgeObjective (objectives.py:132-340), Armijo backtracking
// (optimizers.py:72-121), AdaptiveAlpha (optimizers.py:20-69) and the hard
// result (_make_hard_result, splitters.py:603-690).  The host reads results
// once per level; every control decision (stop rules, line-search retries,
// step-size control, last-feasible tracking, min-side fallback) is made on
// the device.
//
// Work item = (node, group of Rg restarts); one CTA per item (persistent
// queue, largest nodes first).  The restarts of a group share every pass
// over the node's rows:
//   gram pass   : gates pi_r = sigmoid((x.w_r - z_r)/T) and, for all 2*Rg
//                 (restart, side) systems at once, the augmented weighted
//                 Grams sum_k Q[k][c] P[k][e] with P = vech([phi;y][phi;y]^T)
//                 -- one outer-product accumulation in register tiles;
//   solve       : trace-scaled ridge + Cholesky per system (one warp each);
//   resid pass  : loss, envelope gradient [X^T a / T, -sum a / T], n_right;
//   trial pass  : H speculative Armijo step sizes per restart evaluated with
//                 the frozen child models (objectives.py:145-156), accepted in
//                 the reference's order (first passing step of the sequence
//                 alpha0 * rho^k built by repeated multiplication).
// A select kernel then keeps, per node, the best restart as split() does.
#include <algorithm>

#include "bulk.cuh"
#include "common.cuh"
#include "linalg.cuh"
#include "tcgen05.cuh"

namespace art {
namespace {

constexpr int kSplitThreads = 256;
// shared memory of one of two CTAs sharing an SM (228 KB less 1 KB reserved
// per CTA, rounded down)
constexpr size_t kHalfSmem = 110 * 1024;
constexpr int kWarps = kSplitThreads / 32;
constexpr int kMaxCH = 256;      // rows per chunk: a multiple of 32 up to this
constexpr int kMaxP = 64;        // child model features
constexpr int kMaxRg = 16;       // restarts per work item
constexpr int kRedSlots = 5;     // (restart, component) accumulators per thread
constexpr int kBuckets = 64;
constexpr int kMaxStages = 8;    // row-stage ring depth (chunks in flight)
constexpr int kErrSlot = 2 + 2 * kBuckets;  // counts[kErrSlot]: a bounded wait gave up
// Gangs: with at most two restarts per node, a node of n rows is split by
// min(kGangMax, ceil(n / kGangRows)) CTAs that take interleaved chunks and
// add their pass sums in rank order through global scratch.  The gang size
// depends on n alone, so a node's result never depends on its batch.
constexpr int kGangRows = 16384;
constexpr int kGangMax = 16;
// CTA form with FP64 MMA Grams: (side, 8 x 8 block) items per warp, at most
constexpr int kDgMax = 6;
// A gang forms when its last member is popped, which can wait for other
// work items to finish: that wait is bounded by a longer limit than the
// in-pass barriers (members then run side by side).
constexpr uint64_t kGangFormNs = 60ull * 1000000000ull;
// Mixed form, soft passes: the side Grams on the tensor cores.  Chunks of
// kTcRows rows; operand A = the entries P_e = psi_i psi_j of vech([phi; y]
// [phi; y]^T) as 256 M-rows (two M = 128 tiles, entries >= E zero), operand
// B = the weights q_L, q_R of every restart as N = 16 or 32 rows, both TF32
// hi + lo in the K-major core-matrix layout (8 rows x 16 bytes per core
// matrix, no swizzle); D[e][c] = sum_k P_e q_c accumulates in TMEM for
// kTcDrain chunks, then is added into the FP64 Gram in shared memory.
constexpr int kTcRows = 32;
constexpr int kTcEntries = 256;
constexpr int kTcLBO = 128;                          // bytes between K-adjacent core matrices
constexpr int kTcSBO = (kTcRows / 4) * 128;          // bytes between 8-row groups
constexpr int kTcAOp = (kTcEntries / 8) * kTcSBO;    // one A array (hi or lo): 32 KB
constexpr int kTcBOp = (32 / 8) * kTcSBO;            // one B array: 4 KB
constexpr int kTcDrain = 4;
constexpr uint32_t kTcCols = 64;                     // TMEM columns: two tiles x N <= 32

struct SplitArgs {
  int64_t K;
  const int64_t* row_offsets;
  const int64_t* x_offsets;
  const int32_t* dims;
  const int32_t* features;
  const double* x;
  const double* y;
  const double* temperature;
  const double* ridge;
  const double* parent_loss;
  const int8_t* fallback;
  const double* theta0;
  int64_t theta0_stride;
  const uint64_t* node_keys;
  const int32_t* min_side;  // per-node minimum side count or NULL
  ArtSplitParams prm;
  int R, Rg, groups, dmax, pmax, H, TC, S, CH;
  int mixed;  // ART_PRECISION_MIXED: gates in single precision
  int tc;     // mixed form with the soft-pass Grams on the tensor cores
  int dg;     // side Grams as FP64 MMA tiles (8 x 8 blocks of (q psi)^T psi, at most kDgMax per warp)
  // per (node, restart) results, index k * R + r
  double* r_theta;   // [.. ][dmax + 1]
  double* r_loss;
  double* r_beta;    // [..][2][pmax]
  double* r_child;   // [..][2]
  double* r_ridge;   // [..][2]
  int32_t* r_nright;
  int32_t* r_iters;
  int32_t* r_stop;
  int32_t* r_fail;
  int32_t* r_flags;
  int32_t* r_fbiter;
  double* r_alpha;
  double* tr_loss;
  double* tr_step;
  int32_t* tr_back;
  double* tr_gnorm;
  // work queue
  int32_t* counts;   // [0] entries, [1] cursor, [2..2+64) hist, [66..130) start
  int4* items;       // queue entries (item, gang rank, gang size, 0)
  int gang_on, nslots, gang_P;  // gangs enabled; scratch slots; doubles per rank partial
  int4* gang_rec;    // [K * groups]: slot + 1, barrier arrivals, members done, abort
  int32_t* slot_flags;  // [nslots]
  double* gang_scratch; // [nslots][2][kGangMax][gang_P]
};

// Shared-memory layout for a given (dmax, pmax, Rg, H, S, CH): `ring` holds S
// stages of CH rows of x and y (bulk copies in flight), `bars` their
// mbarriers.
struct SLayout {
  size_t ring, rx, rstage, bars, xp, phi, q, G, cache, theta, dirn, grad, lastf, bl, br, trial, red, chol, eidx, rs,
      tcop, tcbar, total;
};
__host__ __device__ inline size_t al(size_t v) { return (v + 15) & ~(size_t)15; }
// phi's row stride: odd, and covering whole 8-column blocks for the MMA Grams
__host__ __device__ inline int phi_stride(int pmax, int dg) {
  const int pa = pmax + 1;
  return dg ? ((8 * ((pa + 7) / 8)) | 1) : (pa | 1);
}
__host__ __device__ inline SLayout split_layout(int dmax, int pmax, int Rg, int H, int S, int CH, int tc = 0,
                                                int dg = 0) {
  SLayout L;
  const int pa = pmax + 1, E = pa * (pa + 1) / 2, dt = dmax + 1;
  size_t o = 0;
  L.rx = al((size_t)CH * dmax * 8 + 32);
  L.rstage = L.rx + al((size_t)CH * 8 + 32);
  L.ring = o; o = al(o + (size_t)S * L.rstage);
  L.bars = o; o = al(o + (size_t)kMaxStages * 8);
  // row-indexed arrays use odd row strides (in doubles), so that lanes
  // reading different rows of a chunk fall in different banks
  L.xp = o; o = al(o + (size_t)CH * (dmax | 1) * 8);
  L.phi = o; o = al(o + (size_t)CH * phi_stride(pmax, dg) * 8);
  L.tcop = 0;
  if (tc) {
    // the weights Q (hard Gram pass), the row cache (residual and trial
    // passes) and the tensor-core operands (soft Gram pass) are never live
    // together: one region, 1 KB aligned for the operand descriptors
    o = (o + 1023) & ~(size_t)1023;
    const size_t qb = (size_t)CH * (2 * Rg + 1) * 8, cb = (size_t)CH * (4 * Rg + 4) * 8;
    const size_t tb = 2 * (size_t)kTcAOp + 2 * (size_t)kTcBOp;
    L.q = L.cache = L.tcop = o;
    o = al(o + (qb > cb ? (qb > tb ? qb : tb) : (cb > tb ? cb : tb)));
  } else {
    L.q = o; o = al(o + (size_t)CH * (2 * Rg + 1) * 8);
  }
  L.G = o; o = al(o + (size_t)E * 2 * Rg * 8);
  if (!tc) { L.cache = o; o = al(o + (size_t)CH * (4 * Rg + 4) * 8); }
  L.theta = o; o = al(o + (size_t)Rg * dt * 8);
  L.dirn = o; o = al(o + (size_t)Rg * dt * 8);
  L.grad = o; o = al(o + (size_t)Rg * dt * 8);
  L.lastf = o; o = al(o + (size_t)Rg * dt * 8);
  L.bl = o; o = al(o + (size_t)Rg * pmax * 8);
  L.br = o; o = al(o + (size_t)Rg * pmax * 8);
  L.trial = o; o = al(o + (size_t)Rg * H * 3 * 8);
  L.red = o; o = al(o + (size_t)Rg * (dmax + 3) * 8);
  L.chol = o; o = al(o + (size_t)kWarps * (E + 2 * pa) * 8);
  L.eidx = o; o = al(o + (size_t)E * 2 * 2);
  L.rs = o; o = al(o + (size_t)Rg * 32 * 8);  // per-restart scalar state
  L.tcbar = 0;
  if (tc) { L.tcbar = o; o = al(o + 16); }  // the MMA completion barrier
  L.total = o;
  return L;
}

// Per-restart scalar state, stored as doubles in smem (slot index below).
enum RS {
  RS_LOSS = 0, RS_DD, RS_TOL, RS_GNORM, RS_T, RS_ALPHA, RS_ASTART, RS_STEP, RS_LSVAL,
  RS_LAML, RS_LAMR, RS_NRIGHT, RS_ACTIVE, RS_ITERS, RS_STOP, RS_FAIL, RS_FAILURES, RS_NBBASE,
  RS_SEARCH, RS_ACCEPT, RS_NB, RS_FEASIT, RS_HASFEAS, RS_CONV, RS_FB, RS_CHOLBAD, RS_HLOSSL,
  RS_HLOSSR, RS_PARENT, RS_INVT, RS_COUNT_
};

// Row groups for a pass: the largest power of two <= 32 such that `items`
// work items times the groups fit the CTA.  Group g of an item takes rows
// g, g + RG, ... of every chunk; the RG threads of an item are consecutive
// lanes of one warp (RG divides 32), so their partials are combined by a
// fixed butterfly of shuffles.
__device__ __forceinline__ int row_groups(int items) {
  int rg = 1;
  while (rg < 32 && items * rg * 2 <= kSplitThreads) rg <<= 1;
  return rg;
}
// Sum over the RG consecutive lanes of a row group (every lane calls).
__device__ __forceinline__ double group_sum(double v, int RG) {
  for (int o = 1; o < RG; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// D = A B + D for one 8 x 8 x 4 FP64 tile (warp-wide): lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma_884(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

struct Item {
  int64_t r0, n, xoff;
  int d, kind, p, pa, E;
  double T0, ridge;
  int k, g, rbase, rn;  // node, group, first restart, restarts in this item
};

__device__ __forceinline__ double sigm(double s) {
  s = fmin(fmax(s, -50.0), 50.0);  // objectives.py:49-51
  return 1.0 / (1.0 + exp(-s));
}

// Mixed form: the gate in single precision with CUDA's fast exponential
// (relative error ~1e-7, inside the form's 1e-5 objective tolerance); the
// score, residuals, solves and every sum stay FP64.
__device__ __forceinline__ double sigm32(double s) {
  const float sf = fminf(fmaxf((float)s, -50.0f), 50.0f);
  return (double)__frcp_rn(1.0f + __expf(-sf));
}

// Entry e of the packed lower triangle -> (i, j), i >= j.
__device__ __forceinline__ void entry_ij(int e, int& i, int& j) {
  i = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
  while (i * (i + 1) / 2 > e) --i;
  while ((i + 1) * (i + 2) / 2 <= e) ++i;
  j = e - i * (i + 1) / 2;
}

// Trace-scaled ridge + left-looking Cholesky + solve of one augmented
// system by a warp: A is the packed lower triangle of [G h; h^T y'Wy]
// (p + 1 rows) in shared memory, overwritten by the factor; the solution
// goes to z[0..p).  lambda = ridge * trace(G) / p (models.py:271).  Returns
// 0, or the 1-based failing pivot.
__device__ __noinline__ int warp_ridge_solve(double* A, double* z, int p, double ridge, double& lam_out) {
  const int lane = threadIdx.x & 31;
  double tr = 0.0;
  if (lane == 0)
    for (int i = 0; i < p; ++i) tr += A[pk(i, i)];
  tr = __shfl_sync(0xffffffffu, tr, 0);
  const double lam = ridge * tr / p;
  lam_out = lam;
  for (int i = lane; i < p; i += 32) A[pk(i, i)] += lam;
  __syncwarp();
  int fail = 0;
  for (int j = 0; j < p && !fail; ++j) {
    double s = 0.0;
    for (int k2 = lane; k2 < j; k2 += 32) s += A[pk(j, k2)] * A[pk(j, k2)];
    s = warp_sum(s);
    const double djj = A[pk(j, j)] - s;
    if (!(djj > 0.0) || !isfinite(djj)) { fail = j + 1; break; }
    const double ljj = sqrt(djj);
    __syncwarp();
    if (lane == 0) A[pk(j, j)] = ljj;
    for (int i = j + 1 + lane; i < p; i += 32) {
      double t2 = A[pk(i, j)];
      for (int k2 = 0; k2 < j; ++k2) t2 -= A[pk(i, k2)] * A[pk(j, k2)];
      A[pk(i, j)] = t2 / ljj;
    }
    __syncwarp();
  }
  if (fail) {
    __syncwarp();
    return fail;
  }
  for (int i = lane; i < p; i += 32) z[i] = A[pk(p, i)];  // h
  __syncwarp();
  warp_forward<double, double>(A, z, p);
  warp_backward<double, double>(A, z, p);
  __syncwarp();
  return 0;
}

// =========================================================== plan (LPT order)
__device__ __forceinline__ int gang_size(const SplitArgs& a, int64_t n) {
  if (!a.gang_on) return 1;
  return (int)min((int64_t)kGangMax, max((int64_t)1, (n + kGangRows - 1) / kGangRows));
}
__global__ void split_plan_hist(SplitArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.K * a.groups) return;
  const int64_t k = t / a.groups;
  const int64_t n = a.row_offsets[k + 1] - a.row_offsets[k];
  const int b = kBuckets - 1 - max(0, min(kBuckets - 1, ilogb((double)(n + 1))));
  atomicAdd(&a.counts[2 + b], gang_size(a, n));
}
__global__ void split_plan_scan(SplitArgs a) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int b = 0; b < kBuckets; ++b) {
    a.counts[2 + kBuckets + b] = c;
    c += a.counts[2 + b];
  }
  a.counts[0] = c;
  a.counts[1] = 0;
}
__global__ void split_plan_scatter(SplitArgs a) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.K * a.groups) return;
  const int64_t k = t / a.groups;
  const int64_t n = a.row_offsets[k + 1] - a.row_offsets[k];
  const int b = kBuckets - 1 - max(0, min(kBuckets - 1, ilogb((double)(n + 1))));
  const int G = gang_size(a, n);
  // a gang's members take consecutive entries, so they are popped together
  const int slot = atomicSub(&a.counts[2 + b], G) - G;
  const int base = a.counts[2 + kBuckets + b] + slot;
  for (int r = 0; r < G; ++r) a.items[base + r] = make_int4((int)t, r, G, 0);
}

// ================================================================ kernel
template <int TC, int TCG>
struct SplitCta {
  static constexpr int TE = 32 / TC;
  const SplitArgs& a;
  unsigned char* sm;
  SLayout L;
  Item it;
  uint64_t* rbar;
  uint32_t rpar = 0, rbusy = 0;  // per-stage wait parity / copy in flight (uniform)
  bool rabort = false;
  // gang of this item: member rank, size, scratch slot, reductions so far
  int grank = 0, gsize = 1, gslot = -1, gpass = 0;
  int64_t gitem = 0;
  const double *xs, *ys;
  double *xp, *phi, *Q, *G, *cache, *th, *dn, *gr, *lf, *bl, *br, *trial, *red, *chol, *rs;
  int xps, phs, qs;  // padded row strides of xp, phi, Q (odd, in doubles)
  int16_t* eidx;
  int tid, lane, warp;

  // tensor-core Gram state: MMA commits issued / waited on the barrier, TMEM base
  uint32_t tc_commits = 0, tc_waits = 0, tmem = 0;

  __device__ SplitCta(const SplitArgs& a_, unsigned char* sm_) : a(a_), sm(sm_) {
    L = split_layout(a.dmax, a.pmax, a.Rg, a.H, a.S, a.CH, a.tc, a.dg);
    rbar = (uint64_t*)(sm + L.bars);
    xs = (const double*)(sm + L.ring); ys = xs; phi = (double*)(sm + L.phi);
    xp = (double*)(sm + L.xp);
    qs = 2 * a.Rg + 1;
    Q = (double*)(sm + L.q); G = (double*)(sm + L.G); cache = (double*)(sm + L.cache);
    th = (double*)(sm + L.theta); dn = (double*)(sm + L.dirn); gr = (double*)(sm + L.grad);
    lf = (double*)(sm + L.lastf); bl = (double*)(sm + L.bl); br = (double*)(sm + L.br);
    trial = (double*)(sm + L.trial); red = (double*)(sm + L.red); chol = (double*)(sm + L.chol);
    eidx = (int16_t*)(sm + L.eidx); rs = (double*)(sm + L.rs);
    tid = threadIdx.x; lane = tid & 31; warp = tid >> 5;
  }
  __device__ double& S(int r, int slot) { return rs[r * 32 + slot]; }
  __device__ double gate(double s) const { return a.mixed ? sigm32(s) : sigm(s); }
  __device__ int dt() const { return it.d + 1; }

  // Row-stage ring: chunk ci of the current node goes to stage ci % S by
  // 1-D bulk copies of its x and y rows; every pass over the rows primes S
  // chunks and refills a stage as soon as the pass is done with it, so
  // copies run S chunks ahead of the arithmetic.  Control flow is uniform:
  // every thread tracks the same parity/in-flight bits; thread 0 issues.
  __device__ void ring_issue(int64_t ci, int st) {
    if (tid == 0) {
      const int64_t c0 = ci * a.CH;
      const int rows = (int)min((int64_t)a.CH, it.n - c0);
      Granules gx = granules(a.x + it.xoff + c0 * it.d, (uint64_t)rows * it.d * 8);
      Granules gy = granules(a.y + it.r0 + c0, (uint64_t)rows * 8);
      unsigned char* base = sm + L.ring + (size_t)st * L.rstage;
      mbar_arrive_expect_tx(&rbar[st], gx.bytes + gy.bytes);
      bulk_g2s(base, gx.base, gx.bytes, &rbar[st]);
      bulk_g2s(base + L.rx, gy.base, gy.bytes, &rbar[st]);
    }
    rbusy |= 1u << st;
  }
  // A gang member takes chunks grank, grank + gsize, ...; its j-th chunk
  // goes to stage j % S.
  __device__ void begin_pass() {
    if (rabort) return;
    for (int j = 0; j < a.S; ++j) {
      const int64_t ci = grank + (int64_t)j * gsize;
      if (ci * a.CH >= it.n) break;
      ring_issue(ci, j);
    }
  }
  // bounded waits for copies still in flight (only after a wait gave up)
  __device__ void ring_drain() {
    for (int st = 0; st < a.S; ++st)
      if (rbusy & (1u << st)) {
        mbar_wait(&rbar[st], (rpar >> st) & 1u);
        rpar ^= 1u << st;
        rbusy &= ~(1u << st);
      }
  }

  // Gang sum of arr[0..len): every member publishes its partial, waits for
  // the others (bounded) and adds all partials in rank order, so every
  // member holds the same total.  Partials alternate between two buffers;
  // a member can only reuse one after passing the next barrier, which the
  // others reach only after reading it.
  __device__ void gang_reduce(double* arr, int len) {
    if (gsize == 1) return;
    __shared__ int s_gok;
    int4* rec = a.gang_rec + gitem;
    const int buf = gpass & 1;
    ++gpass;
    double* base = a.gang_scratch + (size_t)(gslot * 2 + buf) * kGangMax * a.gang_P;
    for (int i = tid; i < len; i += kSplitThreads) __stcg(base + (size_t)grank * a.gang_P + i, arr[i]);
    __threadfence();  // each writer's partial is visible device-wide before the arrival
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(&rec->y, 1);
      const int target = gpass * gsize;
      const uint64_t t0 = globaltimer_ns();
      int ok = 1;
      for (uint32_t spin = 0;; ++spin) {
        if (atomicAdd(&rec->y, 0) >= target) break;
        if (atomicAdd(&rec->w, 0) != 0 || ((spin & 63u) == 63u && globaltimer_ns() - t0 > kWaitNs)) {
          ok = 0;
          break;
        }
      }
      if (!ok) {
        atomicExch(&rec->w, 1);
        atomicExch(&a.counts[kErrSlot], 1);
      }
      __threadfence();
      s_gok = ok;
    }
    __syncthreads();
    if (!s_gok) rabort = true;
    for (int i = tid; i < len; i += kSplitThreads) {
      double v = 0.0;
      for (int r = 0; r < gsize; ++r) v += __ldcg(base + (size_t)r * a.gang_P + i);
      arr[i] = v;
    }
    __syncthreads();
  }

  // Rows [c0, c0 + rows) of x and y from the ring, then the augmented
  // features.  The caller's loop ends every chunk with __syncthreads().
  __device__ int load_chunk(int64_t c0) {
    const int rows = (int)min((int64_t)a.CH, it.n - c0);
    const int d = it.d;
    const int64_t ci = c0 / a.CH;
    const int64_t jj = (ci - grank) / gsize;
    const int st = (int)(jj % a.S);
    if (!rabort) {
      if (jj >= 1) {
        const int64_t cn = grank + (jj - 1 + a.S) * gsize;
        if (cn * a.CH < it.n) ring_issue(cn, (int)((jj - 1) % a.S));
      }
      const bool ok = mbar_wait(&rbar[st], (rpar >> st) & 1u);
      if (ok) {
        rpar ^= 1u << st;
        rbusy &= ~(1u << st);
      }
      if (!__syncthreads_and(ok)) {
        rabort = true;
        if (tid == 0) atomicExch(&a.counts[kErrSlot], 1);
      }
    }
    const unsigned char* base = sm + L.ring + (size_t)st * L.rstage;
    xs = (const double*)(base + (((uintptr_t)(a.x + it.xoff + c0 * d)) & 15));
    ys = (const double*)(base + L.rx + (((uintptr_t)(a.y + it.r0 + c0)) & 15));
    const int pa = it.pa;
    for (int e = tid; e < rows * d; e += kSplitThreads) {
      const int r = e / d, i = e - r * d;
      xp[r * xps + i] = xs[e];
    }
    for (int e = tid; e < rows * pa; e += kSplitThreads) {
      const int r = e / pa, f = e - r * pa;
      double v;
      if (f == it.p) v = ys[r];
      else {
        int ia, ib;
        feature_factors(d, it.kind, f, ia, ib);
        const double* xr = xs + r * d;
        v = (ia < 0 ? 1.0 : xr[ia]) * (ib < 0 ? 1.0 : xr[ib]);
      }
      phi[r * phs + f] = v;
    }
    __syncthreads();
    return rows;
  }

  __device__ double score(int r, int row) {  // x . w_r
    const double* xr = xp + row * xps;
    const double* w = th + r * dt();
    double u0 = 0.0, u1 = 0.0;
    int i = 0;
    for (; i + 1 < it.d; i += 2) {
      u0 = fma(xr[i], w[i], u0);
      u1 = fma(xr[i + 1], w[i + 1], u1);
    }
    if (i < it.d) u0 = fma(xr[i], w[i], u0);
    return u0 + u1;
  }
  __device__ double fitted(const double* beta, int row) {
    const double* pr = phi + row * phs;
    double s0 = 0.0, s1 = 0.0;
    int f = 0;
    for (; f + 1 < it.p; f += 2) {
      s0 = fma(pr[f], beta[f], s0);
      s1 = fma(pr[f + 1], beta[f + 1], s1);
    }
    if (f < it.p) s0 = fma(pr[f], beta[f], s0);
    return s0 + s1;
  }

  // ---- Gram pass on the FP64 tensor path: G_c = (Q[:, c] psi)^T psi over
  // the rows, as lower 8 x 8 blocks (I, J) of NB = ceil((pmax + 1) / 8) block
  // rows, one mma.sync.m8n8k4 per 4 rows.  The (column c, block) items are
  // dealt to the warps (item t to warp t % 8, at most kDgMax each); lane
  // (m, k) of a warp holds rows 8 I + m, columns 8 J + 2 k + {0, 1}.  The
  // gates are computed as in gram_pass.
  __device__ void gram_pass_dg(bool hard) {
    const int C2 = 2 * a.Rg;
    const int NB = (a.pmax + 1 + 7) >> 3, NBLK = NB * (NB + 1) / 2;
    const int nitems = C2 * NBLK;
    const int kq = lane & 3, mq = lane >> 2;
    int code[kDgMax];  // c | I << 8 | J << 16, or -1
#pragma unroll
    for (int u = 0; u < kDgMax; ++u) {
      const int t = warp + kWarps * u;
      code[u] = -1;
      if (t < nitems) {
        const int c = t / NBLK, b = t - c * NBLK;
        int I = 0;
        while ((I + 1) * (I + 2) / 2 <= b) ++I;
        const int J = b - I * (I + 1) / 2;
        code[u] = c | (I << 8) | (J << 16);
      }
    }
    double acc[kDgMax][2];
#pragma unroll
    for (int u = 0; u < kDgMax; ++u) acc[u][0] = acc[u][1] = 0.0;
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
      const int rows = load_chunk(c0);
      for (int pr = tid; pr < rows * a.Rg; pr += kSplitThreads) {
        const int row = pr / a.Rg, r = pr - row * a.Rg;
        double qL = 0.0, qR = 0.0;
        if (r < it.rn && S(r, RS_ACTIVE) != 0.0) {
          if (hard) {
            const double* w = th + r * dt();
            const bool right = right_side(xp + row * xps, w, it.d, w[it.d]);
            qL = right ? 0.0 : 1.0;
            qR = right ? 1.0 : 0.0;
            if (right) atomicAdd(&S(r, RS_NRIGHT), 1.0);  // integers: exact in any order
          } else {
            const double pi = gate((score(r, row) - th[r * dt() + it.d]) * S(r, RS_INVT));
            qL = fmax(1.0 - pi, a.prm.weight_floor);
            qR = fmax(pi, a.prm.weight_floor);
          }
        }
        Q[row * qs + 2 * r] = qL;
        Q[row * qs + 2 * r + 1] = qR;
      }
      __syncthreads();
      for (int k0 = 0; k0 < rows; k0 += 4) {
        const int row = k0 + kq;
        const bool in = row < rows;
        const double* prow = phi + row * phs + mq;
#pragma unroll
        for (int u = 0; u < kDgMax; ++u) {
          if (code[u] >= 0) {  // warp-uniform
            const int c = code[u] & 0xff, I = (code[u] >> 8) & 0xff, J = code[u] >> 16;
            const double av = in ? Q[row * qs + c] * prow[8 * I] : 0.0;
            const double bv = in ? prow[8 * J] : 0.0;
            dmma_884(acc[u], av, bv);
          }
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < kDgMax; ++u) {
      if (code[u] >= 0) {
        const int c = code[u] & 0xff, I = (code[u] >> 8) & 0xff, J = code[u] >> 16;
#pragma unroll
        for (int t2 = 0; t2 < 2; ++t2) {
          const int i = 8 * I + mq, j = 8 * J + 2 * kq + t2;
          if (i < it.pa && j <= i) G[(size_t)pk(i, j) * C2 + c] = acc[u][t2];
        }
      }
    }
    __syncthreads();
    if (gsize > 1) {
      gang_reduce(G, it.E * C2);
      if (hard) {  // right-side counts (integers: exact in any order)
        if (tid < a.Rg) red[tid] = S(tid, RS_NRIGHT);
        __syncthreads();
        gang_reduce(red, a.Rg);
        if (tid < a.Rg) S(tid, RS_NRIGHT) = red[tid];
        __syncthreads();
      }
    }
  }

  // ---- Gram pass: G[e][c] = sum_k Q[k][c] P[k][e]; hard = gates from the
  // exact side of each row (weights 1/0, no floor), else soft gates.
  // Threads beyond the tiles share their rows: RG row groups, group g taking
  // rows g, g + RG, ... of every chunk; the group partials are added in
  // group order at the end (RG = 1, one thread per tile, when the tiles
  // already fill the CTA).
  __device__ void gram_pass(bool hard) {
    if (a.dg) {
      gram_pass_dg(hard);
      return;
    }
    const int E = it.E, C2 = 2 * a.Rg;
    const int nct = (C2 + TC - 1) / TC, net = (E + TE - 1) / TE;
    const int ntiles = nct * net;
    const int RG = row_groups(ntiles);
    const int tile = tid / RG, grp = tid % RG;
    const bool mine = tile < ntiles;
    const int ct = tile % nct, et = tile / nct;
    int ei[TE], ej[TE];
#pragma unroll
    for (int u = 0; u < TE; ++u) {
      const int e = et * TE + u;
      if (mine && e < E) { ei[u] = eidx[2 * e]; ej[u] = eidx[2 * e + 1]; }
      else { ei[u] = 0; ej[u] = 0; }
    }
    double acc[TE][TC];
#pragma unroll
    for (int u = 0; u < TE; ++u)
#pragma unroll
      for (int v = 0; v < TC; ++v) acc[u][v] = 0.0;
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
      const int rows = load_chunk(c0);
      for (int pr = tid; pr < rows * a.Rg; pr += kSplitThreads) {
        const int row = pr / a.Rg, r = pr - row * a.Rg;
        double qL = 0.0, qR = 0.0;
        if (r < it.rn && S(r, RS_ACTIVE) != 0.0) {
          if (hard) {
            const double* w = th + r * dt();
            const bool right = right_side(xp + row * xps, w, it.d, w[it.d]);
            qL = right ? 0.0 : 1.0;
            qR = right ? 1.0 : 0.0;
            // integer-valued sums below 2^53 are exact in any order
            if (right) atomicAdd(&S(r, RS_NRIGHT), 1.0);
          } else {
            const double pi = gate((score(r, row) - th[r * dt() + it.d]) * S(r, RS_INVT));
            qL = fmax(1.0 - pi, a.prm.weight_floor);
            qR = fmax(pi, a.prm.weight_floor);
          }
        }
        Q[row * qs + 2 * r] = qL;
        Q[row * qs + 2 * r + 1] = qR;
      }
      __syncthreads();
      if (mine) {
        for (int row = grp; row < rows; row += RG) {
          const double* pr = phi + row * phs;
          const double* qr = Q + row * qs + ct * TC;
          double pv[TE], qv[TC];
#pragma unroll
          for (int u = 0; u < TE; ++u) pv[u] = pr[ei[u]] * pr[ej[u]];
#pragma unroll
          for (int v = 0; v < TC; ++v) qv[v] = (ct * TC + v < C2) ? qr[v] : 0.0;
#pragma unroll
          for (int u = 0; u < TE; ++u)
#pragma unroll
            for (int v = 0; v < TC; ++v) acc[u][v] = fma(pv[u], qv[v], acc[u][v]);
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < TE; ++u)
#pragma unroll
      for (int v = 0; v < TC; ++v) acc[u][v] = group_sum(acc[u][v], RG);
    if (mine && grp == 0) {
#pragma unroll
      for (int u = 0; u < TE; ++u)
#pragma unroll
        for (int v = 0; v < TC; ++v) {
          const int e = et * TE + u, c = ct * TC + v;
          if (e < E && c < C2) G[(size_t)e * C2 + c] = acc[u][v];
        }
    }
    __syncthreads();
    if (gsize > 1) {
      gang_reduce(G, E * C2);
      if (hard) {  // right-side counts (integers: exact in any order)
        if (tid < a.Rg) red[tid] = S(tid, RS_NRIGHT);
        __syncthreads();
        gang_reduce(red, a.Rg);
        if (tid < a.Rg) S(tid, RS_NRIGHT) = red[tid];
        __syncthreads();
      }
    }
  }

  // Bounded wait for every MMA committed so far.
  __device__ bool tc_wait_all() {
    uint64_t* bar = (uint64_t*)(sm + L.tcbar);
    bool ok = true;
    while (ok && tc_waits < tc_commits) {
      ok = mbar_wait(bar, tc_waits & 1u);
      if (ok) ++tc_waits;
    }
    return ok;
  }

  // ---- soft Gram pass on the tensor cores (mixed form).  Same sums as
  // gram_pass(false): for every (restart, side) column c, G[c][e] =
  // sum_k q_c(k) P_e(k), stored column-major (G + c * E) for solve_all.
  // Gates: FP64 scores, single-precision logistic pair q_R = sigma(s),
  // q_L = sigma(-s) (each accurate relative to itself, so a side with small
  // weights keeps its precision), floored as in the FP64 form.  Products
  // P_e = psi_i psi_j in FP64, split into TF32 hi + lo; three tensor-core
  // products hi hi + hi lo + lo hi per K-step, FP32 accumulation in TMEM over
  // kTcDrain chunks (128 rows), FP64 accumulation across drains.
  __device__ void gram_pass_tc() {
    static_assert(TCG, "the tensor-core pass is compiled into the TCG kernels only");
    const int E = it.E, C2 = 2 * a.Rg, N = C2 <= 16 ? 16 : 32;
    unsigned char* Ahi = sm + L.tcop;
    unsigned char* Alo = Ahi + kTcAOp;
    unsigned char* Bhi = Alo + kTcAOp;
    unsigned char* Blo = Bhi + kTcBOp;
    uint64_t* bar = (uint64_t*)(sm + L.tcbar);
    for (int i = tid; i < E * C2; i += kSplitThreads) G[i] = 0.0;
    // the operand region is shared with the other passes' buffers: the rows
    // no item writes (entries >= E of A, columns >= 2 Rg of B) are cleared
    // here, in both hi and lo, for all 8 K-adjacent core matrices
    for (int i = tid; i < (kTcEntries - E) * 8; i += kSplitThreads) {
      const int e = E + i / 8, kc = i % 8;
      const size_t off = (size_t)(e >> 3) * kTcSBO + (size_t)kc * 128 + (size_t)(e & 7) * 16;
      *(uint4*)(Ahi + off) = make_uint4(0, 0, 0, 0);
      *(uint4*)(Alo + off) = make_uint4(0, 0, 0, 0);
    }
    for (int i = tid; i < (N - C2) * 8; i += kSplitThreads) {
      const int c = C2 + i / 8, kc = i % 8;
      const size_t off = (size_t)(c >> 3) * kTcSBO + (size_t)kc * 128 + (size_t)(c & 7) * 16;
      *(uint4*)(Bhi + off) = make_uint4(0, 0, 0, 0);
      *(uint4*)(Blo + off) = make_uint4(0, 0, 0, 0);
    }
    const uint32_t idesc = idesc_tf32(128, N);
    const int nB = a.Rg * (kTcRows / 8), nA = E * (kTcRows / 8);
    int64_t chunk = 0;  // sub-chunks of kTcRows rows issued in this pass
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
     const int crows = load_chunk(c0);
     for (int sub = 0; sub * kTcRows < crows; ++sub, ++chunk) {
      const int r0 = sub * kTcRows;
      const int rows = min(kTcRows, crows - r0);
      const bool last = c0 + (int64_t)gsize * a.CH >= it.n && r0 + kTcRows >= crows;
      // the operand buffers are free once every earlier MMA has completed
      const bool okw = tc_wait_all();
      if (!__syncthreads_and(okw)) {
        rabort = true;
        if (tid == 0) atomicExch(&a.counts[kErrSlot], 1);
      }
      // items: (restart, octet of rows) -> gates; (entry, octet) -> products
      for (int j = tid; j < nB + nA; j += kSplitThreads) {
        if (j < nB) {
          const int r = j / (kTcRows / 8), oct = j - r * (kTcRows / 8);
          uint32_t lh[8], ll[8], rh[8], rl[8];
          const bool on = r < it.rn && S(r, RS_ACTIVE) != 0.0;
          const double invt = S(r, RS_INVT), z = th[r * dt() + it.d];
#pragma unroll
          for (int e8 = 0; e8 < 8; ++e8) {
            const int row = oct * 8 + e8;
            float qL = 0.0f, qR = 0.0f;
            if (on && row < rows) {
              const float sf = fminf(fmaxf((float)((score(r, r0 + row) - z) * invt), -50.0f), 50.0f);
              const float en = __expf(-sf);
              qR = __frcp_rn(1.0f + en);
              qL = en * qR;
              qR = fmaxf(qR, (float)a.prm.weight_floor);
              qL = fmaxf(qL, (float)a.prm.weight_floor);
            }
            lh[e8] = to_tf32(qL);
            ll[e8] = to_tf32(qL - __uint_as_float(lh[e8]));
            rh[e8] = to_tf32(qR);
            rl[e8] = to_tf32(qR - __uint_as_float(rh[e8]));
          }
          const int cl = 2 * r, cr = 2 * r + 1;
          const size_t ol = (size_t)(cl >> 3) * kTcSBO + (size_t)(2 * oct) * 128 + (size_t)(cl & 7) * 16;
          const size_t orr = (size_t)(cr >> 3) * kTcSBO + (size_t)(2 * oct) * 128 + (size_t)(cr & 7) * 16;
          *(uint4*)(Bhi + ol) = make_uint4(lh[0], lh[1], lh[2], lh[3]);
          *(uint4*)(Bhi + ol + 128) = make_uint4(lh[4], lh[5], lh[6], lh[7]);
          *(uint4*)(Blo + ol) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
          *(uint4*)(Blo + ol + 128) = make_uint4(ll[4], ll[5], ll[6], ll[7]);
          *(uint4*)(Bhi + orr) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
          *(uint4*)(Bhi + orr + 128) = make_uint4(rh[4], rh[5], rh[6], rh[7]);
          *(uint4*)(Blo + orr) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
          *(uint4*)(Blo + orr + 128) = make_uint4(rl[4], rl[5], rl[6], rl[7]);
        } else {
          const int jj = j - nB;
          const int e = jj % E, oct = jj / E;
          const int fi = eidx[2 * e], fj = eidx[2 * e + 1];
          uint32_t ph[8], pl[8];
#pragma unroll
          for (int e8 = 0; e8 < 8; ++e8) {
            const int row = oct * 8 + e8;
            float v = 0.0f;
            if (row < rows) {
              const double* pr = phi + (r0 + row) * phs;
              v = (float)(pr[fi] * pr[fj]);
            }
            ph[e8] = to_tf32(v);
            pl[e8] = to_tf32(v - __uint_as_float(ph[e8]));
          }
          const size_t off = (size_t)(e >> 3) * kTcSBO + (size_t)(2 * oct) * 128 + (size_t)(e & 7) * 16;
          *(uint4*)(Ahi + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *(uint4*)(Ahi + off + 128) = make_uint4(ph[4], ph[5], ph[6], ph[7]);
          *(uint4*)(Alo + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
          *(uint4*)(Alo + off + 128) = make_uint4(pl[4], pl[5], pl[6], pl[7]);
        }
      }
      fence_proxy_async();  // operand writes -> visible to the tensor core
      __syncthreads();
      const bool fresh = (chunk % kTcDrain) == 0;
      if (tid == 0 && !rabort) {
        tc_fence_after();
        const uint32_t ah = smem_u32(Ahi), alo = smem_u32(Alo), bh = smem_u32(Bhi), blo = smem_u32(Blo);
#pragma unroll
        for (int ks = 0; ks < kTcRows / 8; ++ks) {
          const uint32_t ko = (uint32_t)ks * 2u * kTcLBO;  // 8 rows = two K-adjacent core matrices
#pragma unroll
          for (int prod = 0; prod < 3; ++prod) {
            const uint32_t A = (prod == 2) ? alo : ah;
            const uint32_t B = (prod == 1) ? blo : bh;
            const uint32_t acc = (fresh && ks == 0 && prod == 0) ? 0u : 1u;
#pragma unroll
            for (int t = 0; t < 2; ++t)
              mma_tf32(tmem + (uint32_t)(t * N), smem_desc_kmajor(A + (uint32_t)t * 16u * kTcSBO + ko, kTcLBO, kTcSBO),
                       smem_desc_kmajor(B + ko, kTcLBO, kTcSBO), idesc, acc);
          }
        }
        mma_commit(bar);
      }
      if (!rabort) ++tc_commits;
      const bool seg_end = ((chunk + 1) % kTcDrain) == 0 || last;
      if (seg_end && !rabort) {
        const bool ok = tc_wait_all();
        if (!__syncthreads_and(ok)) {
          rabort = true;
          if (tid == 0) atomicExch(&a.counts[kErrSlot], 1);
        } else {
          tc_fence_after();
          // warps 0-3: tile 0 (entries 0..127); warps 4-7: tile 1 (128..255)
          const int quarter = warp & 3, t = warp >> 2;
          const int e = t * 128 + quarter * 32 + lane;
          const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(t * N);
          for (int cb = 0; cb < N; cb += 16) {
            float v[16];
            tmem_ld16(lane_base + (uint32_t)cb, v);
            if (e < E) {
#pragma unroll
              for (int q = 0; q < 16; ++q)
                if (cb + q < C2) G[(size_t)(cb + q) * E + e] += (double)v[q];
            }
          }
          tc_fence_before();
        }
      }
      __syncthreads();
     }
    }
    // every MMA of the pass has been drained: the operand region is free for
    // the row cache of the next passes
    if (gsize > 1) gang_reduce(G, E * C2);
  }

  // ---- trace-scaled ridge + Cholesky + solve for every (restart, side).
  // One warp per system; a failed factorisation marks the restart.
  // `colmajor`: the Grams are stored G[c * E + e] (tensor-core pass) instead
  // of G[e * C2 + c].
  __device__ void solve_all(bool colmajor = false) {
    const int p = it.p, pa = it.pa, E = it.E, C2 = 2 * a.Rg;
    double* A = chol + (size_t)warp * (E + 2 * pa);
    double* z = A + E;
    for (int c = warp; c < 2 * it.rn; c += kWarps) {
      const int r = c >> 1, side = c & 1;
      if (S(r, RS_ACTIVE) == 0.0) continue;
      for (int e = lane; e < E; e += 32) A[e] = colmajor ? G[(size_t)c * E + e] : G[(size_t)e * C2 + c];
      __syncwarp();
      double lam;
      const int fail = warp_ridge_solve(A, z, p, it.ridge, lam);
      if (fail) {
        if (lane == 0) S(r, RS_CHOLBAD) = 1.0;
        __syncwarp();
        continue;
      }
      double* beta = (side ? br : bl) + r * a.pmax;
      for (int i = lane; i < p; i += 32) beta[i] = z[i];
      if (lane == 0) S(r, side ? RS_LAMR : RS_LAML) = lam;
      __syncwarp();
    }
    __syncthreads();
  }

  // ---- soft residual pass: loss, gradient, n_right for active restarts.
  __device__ void resid_pass() {
    const int d = it.d, comps = d + 3;  // grad_w (d), sum a, loss, n_right
    const int pairs = a.Rg * comps;
    // few (restart, component) pairs: RGr row groups share each pair (as in
    // gram_pass), combined in group order at the end; otherwise one thread
    // per pair over kRedSlots slots
    const int RGr = pairs <= kSplitThreads ? row_groups(pairs) : 1;
    const int gq = tid / RGr, ggrp = tid % RGr;
    double accs[kRedSlots];
#pragma unroll
    for (int s = 0; s < kRedSlots; ++s) accs[s] = 0.0;
    const int cst = a.Rg + 1;                  // padded row stride
    const double inv_n = 1.0 / (double)it.n;
    double* coef = cache;                      // [row][r]: a_k
    double* wl = cache + a.CH * cst;           // [row][r]: weighted loss term
    double* nr = cache + 2 * a.CH * cst;       // [row][r]: pi >= 0.5
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
      const int rows = load_chunk(c0);
      for (int pr = tid; pr < rows * a.Rg; pr += kSplitThreads) {
        const int row = pr / a.Rg, r = pr - row * a.Rg;
        double cf = 0.0, lw = 0.0, ge = 0.0;
        if (r < it.rn && S(r, RS_ACTIVE) != 0.0) {
          const double pi = gate((score(r, row) - th[r * dt() + d]) * S(r, RS_INVT));
          const double yv = ys[row];
          const double eL = yv - fitted(bl + r * a.pmax, row);
          const double eR = yv - fitted(br + r * a.pmax, row);
          const double eL2 = eL * eL, eR2 = eR * eR;
          lw = (1.0 - pi) * eL2 + pi * eR2;
          cf = (eR2 - eL2) * pi * (1.0 - pi) * inv_n;
          ge = pi >= 0.5 ? 1.0 : 0.0;
        }
        coef[row * cst + r] = cf;
        wl[row * cst + r] = lw;
        nr[row * cst + r] = ge;
      }
      __syncthreads();
      if (RGr > 1) {
        if (gq < pairs) {
          const int r = gq / comps, cp = gq - r * comps;
          double acc = accs[0];
          for (int row = ggrp; row < rows; row += RGr) {
            const double cv = coef[row * cst + r];
            if (cp < d) acc = fma(cv, xp[row * xps + cp], acc);
            else if (cp == d) acc += cv;
            else if (cp == d + 1) acc += wl[row * cst + r];
            else acc += nr[row * cst + r];
          }
          accs[0] = acc;
        }
      } else {
#pragma unroll
      for (int s = 0; s < kRedSlots; ++s) {
        const int q = tid + s * kSplitThreads;
        if (q < pairs) {
          const int r = q / comps, cp = q - r * comps;
          double acc = accs[s];
          for (int row = 0; row < rows; ++row) {
            const double cv = coef[row * cst + r];
            if (cp < d) acc = fma(cv, xp[row * xps + cp], acc);
            else if (cp == d) acc += cv;
            else if (cp == d + 1) acc += wl[row * cst + r];
            else acc += nr[row * cst + r];
          }
          accs[s] = acc;
        }
      }
      }
      __syncthreads();
    }
    if (RGr > 1) {
      const double tot = group_sum(accs[0], RGr);
      if (gq < pairs && ggrp == 0) red[gq] = tot;
      __syncthreads();
    } else {
#pragma unroll
      for (int s = 0; s < kRedSlots; ++s) {
        const int q = tid + s * kSplitThreads;
        if (q < pairs) red[q] = accs[s];
      }
      __syncthreads();
    }
    gang_reduce(red, pairs);
    // finalize per restart (one thread each)
    if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0) {
      const int r = tid;
      const double T = S(r, RS_T);
      const double* rr = red + r * comps;
      double* g = gr + r * dt();
      for (int i = 0; i < d; ++i) g[i] = rr[i] / T;
      g[d] = -rr[d] / T;
      S(r, RS_LOSS) = rr[d + 1] / (double)it.n;
      S(r, RS_NRIGHT) = rr[d + 2];
      // projected gradient and its norm (splitters.py:86-98)
      const double* w = th + r * dt();
      double gw = 0.0;
      for (int i = 0; i < d; ++i) gw += g[i] * w[i];
      double* pd = dn + r * dt();
      double nrm2 = 0.0;
      for (int i = 0; i < d; ++i) {
        const double pg = g[i] - gw * w[i];
        pd[i] = -pg;
        nrm2 += pg * pg;
      }
      pd[d] = -g[d];
      nrm2 += g[d] * g[d];
      S(r, RS_GNORM) = sqrt(nrm2);
      double dd = 0.0;
      for (int i = 0; i <= d; ++i) dd += g[i] * pd[i];
      S(r, RS_DD) = dd;
    }
    __syncthreads();
  }

  // ---- trial pass: frozen-model losses of H step sizes per searching restart.
  __device__ void trial_pass() {
    const int d = it.d, H = a.H;
    double* tal = trial;                       // [r][H] alpha
    double* tnr = trial + a.Rg * H;            // [r][H] ||w + alpha p_w||
    double* tf = trial + 2 * a.Rg * H;         // [r][H] accumulated loss
    // row groups as in gram_pass: RG threads share each (restart, step) item
    const int items = a.Rg * H;
    const int RG = row_groups(items);
    const int item = tid / RG, grp = tid % RG;
    const bool mine = item < items;
    const int r = item / H, j = item - (item / H) * H;
    double f = 0.0;
    const bool on = mine && r < it.rn && S(r, RS_SEARCH) != 0.0;
    double alpha = 0.0, inv_nrm = 1.0, z = 0.0, pz = 0.0, inv_t = 1.0;
    if (on) {
      alpha = tal[r * H + j];
      inv_nrm = 1.0 / tnr[r * H + j];
      z = th[r * dt() + d];
      pz = dn[r * dt() + d];
      inv_t = S(r, RS_INVT);
    }
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
      const int rows = load_chunk(c0);
      for (int pr = tid; pr < rows * a.Rg; pr += kSplitThreads) {
        const int row = pr / a.Rg, rr = pr - row * a.Rg;
        double* cp = cache + row * (4 * a.Rg + 1) + rr * 4;
        if (rr < it.rn && S(rr, RS_SEARCH) != 0.0) {
          const double* xr = xp + row * xps;
          const double* w = th + rr * dt();
          const double* pw = dn + rr * dt();
          double u = 0.0, v = 0.0, u1 = 0.0, v1 = 0.0;
          int i = 0;
          for (; i + 1 < d; i += 2) {
            u = fma(xr[i], w[i], u);
            v = fma(xr[i], pw[i], v);
            u1 = fma(xr[i + 1], w[i + 1], u1);
            v1 = fma(xr[i + 1], pw[i + 1], v1);
          }
          if (i < d) { u = fma(xr[i], w[i], u); v = fma(xr[i], pw[i], v); }
          u += u1;
          v += v1;
          const double yv = ys[row];
          const double eL = yv - fitted(bl + rr * a.pmax, row);
          const double eR = yv - fitted(br + rr * a.pmax, row);
          cp[0] = u; cp[1] = v; cp[2] = eL * eL; cp[3] = eR * eR;
        }
      }
      __syncthreads();
      if (on) {
        for (int row = grp; row < rows; row += RG) {
          const double* cp = cache + row * (4 * a.Rg + 1) + r * 4;
          const double s = ((cp[0] + alpha * cp[1]) * inv_nrm - (z + alpha * pz)) * inv_t;
          const double pi = gate(s);
          f += (1.0 - pi) * cp[2] + pi * cp[3];
        }
      }
      __syncthreads();
    }
    f = group_sum(f, RG);
    if (on && grp == 0) tf[r * H + j] = f;
    __syncthreads();
    gang_reduce(tf, a.Rg * H);
    if (on && grp == 0) tf[r * H + j] = tf[r * H + j] / (double)it.n;
    __syncthreads();
  }

  __device__ void record_trace(int r, int iter) {
    const int64_t kr = (int64_t)it.k * a.R + it.rbase + r;
    const int M = a.prm.max_iters;
    if (grank != 0) return;
    if (a.tr_loss) a.tr_loss[kr * (M + 1) + iter] = S(r, RS_LOSS);
    if (a.tr_gnorm) a.tr_gnorm[kr * (M + 1) + iter] = S(r, RS_GNORM);
  }

  __device__ void run(int item_id, int rank, int members);
  __device__ bool gang_begin(int item_id, int rank, int members);
  __device__ void gang_end();
};

template <int TC, int TCG>
__device__ bool SplitCta<TC, TCG>::gang_begin(int item_id, int rank, int members) {
  // rank 0 takes a free scratch slot and publishes it; the other members
  // wait (bounded) for it.  At most one gang is being popped at a time and
  // every other active gang holds >= 2 CTAs, so the slots (one per SM plus
  // two) never run out.
  __shared__ int s_slot;
  grank = rank;
  gsize = members;
  gitem = item_id;
  gpass = 0;
  if (members == 1) return true;
  int4* rec = a.gang_rec + item_id;
  if (tid == 0) {
    int slot = -1, taken = -1;  // taken: the slot rank 0 holds, kept after a failed formation
    const uint64_t t0 = globaltimer_ns();
    if (rank == 0) {
      for (uint32_t spin = 0; slot < 0; ++spin) {
        for (int q = 0; q < a.nslots && slot < 0; ++q)
          if (atomicCAS(&a.slot_flags[q], 0, 1) == 0) slot = q;
        if (slot < 0 && (spin & 63u) == 63u && globaltimer_ns() - t0 > kWaitNs) break;
      }
      if (slot >= 0) {
        taken = slot;
        __threadfence();
        atomicExch(&rec->x, slot + 1);
      }
    } else {
      for (uint32_t spin = 0;; ++spin) {
        const int v = atomicAdd(&rec->x, 0);
        if (v > 0) { slot = v - 1; break; }
        if ((spin & 63u) == 63u && globaltimer_ns() - t0 > kWaitNs) break;
      }
      __threadfence();
    }
    // formation: every member arrives once, then waits for all of them
    if (slot >= 0) {
      atomicAdd(&rec->y, 1);
      const uint64_t t1 = globaltimer_ns();
      for (uint32_t spin = 0;; ++spin) {
        if (atomicAdd(&rec->y, 0) >= members) break;
        if (atomicAdd(&rec->w, 0) != 0 ||
            ((spin & 63u) == 63u && globaltimer_ns() - t1 > kGangFormNs)) {
          slot = -1;
          break;
        }
      }
      __threadfence();
    }
    if (slot < 0) {
      atomicExch(&rec->w, 1);
      atomicExch(&a.counts[kErrSlot], 1);
      // the level is lost; give the slot back so later gangs of this launch
      // do not wait out their limits for it
      if (taken >= 0) atomicExch(&a.slot_flags[taken], 0);
    }
    s_slot = slot;
  }
  __syncthreads();
  gslot = s_slot;
  gpass = 1;  // the formation counted as the first barrier
  __syncthreads();
  return gslot >= 0;
}

template <int TC, int TCG>
__device__ void SplitCta<TC, TCG>::gang_end() {
  if (gsize == 1) return;
  __syncthreads();
  if (tid == 0 && gslot >= 0) {
    __threadfence();
    int4* rec = a.gang_rec + gitem;
    if (atomicAdd(&rec->z, 1) == gsize - 1) atomicExch(&a.slot_flags[gslot], 0);
  }
  gsize = 1;
  grank = 0;
  gslot = -1;
}

template <int TC, int TCG>
__device__ void SplitCta<TC, TCG>::run(int item_id, int rank, int members) {
  const ArtSplitParams& P = a.prm;
  if (!gang_begin(item_id, rank, members)) {  // no slot: the level is reported lost
    gang_end();
    return;
  }
  // ---------------------------------------------------------------- setup
  const int k = item_id / a.groups, g = item_id - (item_id / a.groups) * a.groups;
  it.k = k;
  it.g = g;
  it.r0 = a.row_offsets[k];
  it.n = a.row_offsets[k + 1] - it.r0;
  it.xoff = a.x_offsets[k];
  it.d = a.dims[k];
  it.kind = a.features[k];
  it.p = feature_count(it.d, it.kind);
  it.pa = it.p + 1;
  xps = it.d | 1;
  phs = a.dg ? phi_stride(a.pmax, 1) : (it.pa | 1);
  it.E = it.pa * (it.pa + 1) / 2;
  it.T0 = a.temperature[k];
  it.ridge = a.ridge[k];
  it.rbase = g * a.Rg;
  it.rn = min(a.Rg, a.R - it.rbase);
  const int d = it.d, n = (int)it.n;
  const int req = max(a.min_side ? max(1, a.min_side[k]) : P.min_side_points,
                      (int)ceil(P.min_side_fraction * (double)n));
  const bool fb_allowed = a.fallback ? a.fallback[k] != 0 : false;
  for (int e = tid; e < it.E; e += kSplitThreads) {
    int i, j;
    entry_ij(e, i, j);
    eidx[2 * e] = (int16_t)i;
    eidx[2 * e + 1] = (int16_t)j;
  }
  for (int q = tid; q < a.Rg * 32; q += kSplitThreads) rs[q] = 0.0;
  if (a.dg)  // phi's columns past this item's pa read as zeros in the MMA Grams
    for (int e = tid; e < a.CH * phs; e += kSplitThreads) phi[e] = 0.0;
  __syncthreads();
  // initial theta: projected theta0 (splitters.py:379)
  if (tid < it.rn) {
    const int r = tid;
    const int64_t kr = (int64_t)k * a.R + it.rbase + r;
    const double* t0 = a.theta0 + kr * a.theta0_stride;
    double* t = th + r * dt();
    double nrm2 = 0.0;
    for (int i = 0; i < d; ++i) nrm2 += t0[i] * t0[i];
    const double nrm = sqrt(nrm2);
    S(r, RS_ACTIVE) = 1.0;
    if (!(nrm > 1e-12) || !isfinite(nrm)) {
      S(r, RS_ACTIVE) = 0.0;
      S(r, RS_FAIL) = ART_SPLIT_INVALID;
    }
    for (int i = 0; i < d; ++i) t[i] = t0[i] / nrm;
    t[d] = t0[d];
    S(r, RS_T) = it.T0;
    S(r, RS_INVT) = 1.0 / it.T0;
    S(r, RS_ALPHA) = fmin(fmax(P.alpha0, P.alpha_min), P.alpha_max);
    S(r, RS_STOP) = ART_STOP_MAX_ITERS;
    S(r, RS_FEASIT) = -1.0;
  }
  __syncthreads();
  if (n == 0) {  // nothing to split
    if (tid < it.rn) { S(tid, RS_ACTIVE) = 0.0; S(tid, RS_FAIL) = ART_SPLIT_MIN_SIDE_POINTS; }
    __syncthreads();
  }
  // ---------------------------------------------------------- evaluate(theta)
  auto evaluate = [&]() {
    if constexpr (TCG) {
      gram_pass_tc();
      solve_all(true);
    } else {
      gram_pass(false);
      solve_all();
    }
    if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0 && S(tid, RS_CHOLBAD) != 0.0) {
      S(tid, RS_ACTIVE) = 0.0;
      S(tid, RS_FAIL) = ART_SPLIT_CHOLESKY_FAILURE;
    }
    __syncthreads();
    resid_pass();
  };
  evaluate();
  if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0) {
    const int r = tid;
    const double g0 = S(r, RS_GNORM);
    S(r, RS_TOL) = P.grad_atol + P.grad_rtol * g0;
    const int nr = (int)S(r, RS_NRIGHT);
    if (min(nr, n - nr) >= req) {
      S(r, RS_HASFEAS) = 1.0;
      S(r, RS_FEASIT) = 0.0;
      for (int i = 0; i <= d; ++i) lf[r * dt() + i] = th[r * dt() + i];
    }
    record_trace(r, 0);
  }
  __syncthreads();
  // ------------------------------------------------------------------ loop
  for (int iter = 0; iter < P.max_iters; ++iter) {
    // stop checks (splitters.py:424-437)
    if (tid < it.rn) {
      const int r = tid;
      S(r, RS_SEARCH) = 0.0;
      S(r, RS_ACCEPT) = 0.0;
      if (S(r, RS_ACTIVE) != 0.0) {
        if (S(r, RS_GNORM) <= S(r, RS_TOL)) {
          S(r, RS_CONV) = 1.0;
          S(r, RS_STOP) = ART_STOP_GRADIENT_TOLERANCE;
          S(r, RS_ACTIVE) = 0.0;
        } else if (S(r, RS_DD) >= 0.0) {
          S(r, RS_STOP) = ART_STOP_NON_DESCENT;
          S(r, RS_ACTIVE) = 0.0;
        } else {
          S(r, RS_SEARCH) = 1.0;
          S(r, RS_FAILURES) = 0.0;
          S(r, RS_NBBASE) = 0.0;
          S(r, RS_ASTART) = P.adaptive_alpha ? S(r, RS_ALPHA) : P.alpha0;
        }
      }
    }
    __syncthreads();
    // ---------------------------------------------------- line search
    const int max_batches = (P.max_backtracks + 1 + a.H - 1) / a.H * P.max_line_search_failures + 1;
    for (int batch = 0; batch < max_batches; ++batch) {
      int any = 0;
      if (tid < it.rn) any = S(tid, RS_SEARCH) != 0.0;
      if (!__syncthreads_or(any)) break;
      // step sizes alpha0 * rho^k by repeated multiplication (optimizers.py:104-107)
      if (tid < it.rn && S(tid, RS_SEARCH) != 0.0) {
        const int r = tid, H = a.H;
        double al = S(r, RS_ASTART);
        const int base = (int)S(r, RS_NBBASE);
        for (int q = 0; q < base; ++q) al *= P.rho;
        const double* w = th + r * dt();
        const double* pw = dn + r * dt();
        for (int j = 0; j < H; ++j) {
          if (j > 0) al *= P.rho;
          double nrm2 = 0.0;
          for (int i = 0; i < d; ++i) {
            const double v = w[i] + al * pw[i];
            nrm2 += v * v;
          }
          trial[r * H + j] = al;
          trial[a.Rg * H + r * H + j] = sqrt(nrm2);
        }
      }
      __syncthreads();
      trial_pass();
      if (tid < it.rn && S(tid, RS_SEARCH) != 0.0) {
        const int r = tid, H = a.H;
        const int base = (int)S(r, RS_NBBASE);
        const double f0 = S(r, RS_LOSS), dd = S(r, RS_DD);
        int acc_j = -1;
        for (int j = 0; j < H && base + j <= P.max_backtracks; ++j) {
          const double al = trial[r * H + j];
          const double rhs = __dadd_rn(f0, __dmul_rn(__dmul_rn(P.armijo_c, al), dd));
          if (trial[2 * a.Rg * H + r * H + j] <= rhs) { acc_j = j; break; }
        }
        bool attempt_done = false, success = false;
        double step = 0.0;
        int nb = 0;
        if (acc_j >= 0) {
          attempt_done = true;
          success = true;
          step = trial[r * H + acc_j];
          nb = base + acc_j;
          S(r, RS_LSVAL) = trial[2 * a.Rg * H + r * H + acc_j];
        } else if (base + H > P.max_backtracks) {
          attempt_done = true;
          const int last = P.max_backtracks - base;
          step = trial[r * H + last];
          nb = P.max_backtracks;
        } else {
          S(r, RS_NBBASE) = base + H;
        }
        if (attempt_done) {
          if (P.adaptive_alpha) {  // AdaptiveAlpha.update (optimizers.py:49-66)
            double na;
            if (!success) na = step * P.rho;
            else if (nb == 0) na = step * P.alpha_grow;
            else if (nb >= P.heavy_backtrack_threshold) na = step * P.alpha_recovery;
            else na = step / P.rho;
            S(r, RS_ALPHA) = fmin(fmax(na, P.alpha_min), P.alpha_max);
          }
          if (success) {
            S(r, RS_SEARCH) = 0.0;
            S(r, RS_ACCEPT) = 1.0;
            S(r, RS_STEP) = step;
            S(r, RS_NB) = nb;
          } else {
            const double fails = S(r, RS_FAILURES) + 1.0;
            S(r, RS_FAILURES) = fails;
            int stop = -1;
            if (!P.adaptive_alpha) stop = ART_STOP_LINE_SEARCH_FAILED;
            else if (fails >= P.max_line_search_failures) stop = ART_STOP_MAX_LINE_SEARCH_FAILURES;
            else if (S(r, RS_ALPHA) <= P.alpha_min) stop = ART_STOP_ALPHA_MIN_REACHED;
            if (stop >= 0) {
              S(r, RS_STOP) = stop;
              S(r, RS_SEARCH) = 0.0;
              S(r, RS_ACTIVE) = 0.0;
            } else {
              S(r, RS_NBBASE) = 0.0;
              S(r, RS_ASTART) = S(r, RS_ALPHA);
            }
          }
        }
      }
      __syncthreads();
    }
    // restarts still searching after the batch cap stop (cannot happen with
    // the cap above; kept as a bound on device work)
    if (tid < it.rn && S(tid, RS_SEARCH) != 0.0) {
      S(tid, RS_SEARCH) = 0.0;
      S(tid, RS_ACTIVE) = 0.0;
      S(tid, RS_STOP) = ART_STOP_MAX_LINE_SEARCH_FAILURES;
    }
    // commit accepted steps: theta <- project(theta + alpha d) (splitters.py:451, 497)
    int any_acc = 0;
    if (tid < it.rn && S(tid, RS_ACCEPT) != 0.0) {
      any_acc = 1;
      const int r = tid;
      const double al = S(r, RS_STEP);
      double* t = th + r * dt();
      const double* pd = dn + r * dt();
      double nrm2 = 0.0;
      for (int i = 0; i < d; ++i) {
        const double v = t[i] + al * pd[i];
        t[i] = v;
        nrm2 += v * v;
      }
      const double nrm = sqrt(nrm2);
      for (int i = 0; i < d; ++i) t[i] = t[i] / nrm;
      t[d] = t[d] + al * pd[d];
      if (P.anneal_ratio != 1.0 && P.max_iters > 1)
      {
        S(r, RS_T) = it.T0 * pow(P.anneal_ratio, (double)(iter + 1) / (double)(P.max_iters - 1));
        S(r, RS_INVT) = 1.0 / S(r, RS_T);
      }
      S(r, RS_ITERS) = iter + 1;
      const int64_t kr = (int64_t)k * a.R + it.rbase + r;
      if (a.tr_step && grank == 0) a.tr_step[kr * P.max_iters + iter] = al;
      if (a.tr_back && grank == 0) a.tr_back[kr * P.max_iters + iter] = (int)S(r, RS_NB);
    } else if (tid < it.rn) {
      S(tid, RS_ACTIVE) = 0.0;  // stopped this iteration (reason already set)
    }
    if (!__syncthreads_or(any_acc)) break;
    evaluate();
    if (tid < it.rn && S(tid, RS_ACCEPT) != 0.0 && S(tid, RS_ACTIVE) != 0.0) {
      const int r = tid;
      const int nr = (int)S(r, RS_NRIGHT);
      if (min(nr, n - nr) >= req) {
        S(r, RS_HASFEAS) = 1.0;
        S(r, RS_FEASIT) = (double)(iter + 1);
        for (int i = 0; i <= d; ++i) lf[r * dt() + i] = th[r * dt() + i];
      }
      record_trace(r, iter + 1);
    }
    __syncthreads();
  }
  // ------------------------------------------------ finish (splitters.py:584-601)
  if (tid < it.rn) {
    const int r = tid;
    if (S(r, RS_FAIL) == 0.0) {
      S(r, RS_ACTIVE) = 1.0;  // participate in the hard passes
      const int nr = (int)S(r, RS_NRIGHT);
      const bool final_ok = min(nr, n - nr) >= req;
      if (!final_ok && fb_allowed && S(r, RS_HASFEAS) != 0.0) {
        for (int i = 0; i <= d; ++i) th[r * dt() + i] = lf[r * dt() + i];
        S(r, RS_FB) = 1.0;
      }
      // re-project (splitters.py:614)
      double* t = th + r * dt();
      double nrm2 = 0.0;
      for (int i = 0; i < d; ++i) nrm2 += t[i] * t[i];
      const double nrm = sqrt(nrm2);
      for (int i = 0; i < d; ++i) t[i] = t[i] / nrm;
    } else {
      S(r, RS_ACTIVE) = 0.0;
    }
    S(r, RS_CHOLBAD) = 0.0;
  }
  __syncthreads();
  // hard partition: exact sides, right-side counts and (for refits) the hard Grams
  if (tid < it.rn) S(tid, RS_NRIGHT) = 0.0;
  __syncthreads();
  gram_pass(true);
  if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0) {
    const int nr = (int)S(tid, RS_NRIGHT);
    if (nr < req || n - nr < req) {
      S(tid, RS_ACTIVE) = 0.0;
      S(tid, RS_FAIL) = ART_SPLIT_MIN_SIDE_POINTS;
    }
  }
  __syncthreads();
  if (P.hard_refit) {
    solve_all();  // hard child models from the hard Grams
    if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0 && S(tid, RS_CHOLBAD) != 0.0) {
      S(tid, RS_ACTIVE) = 0.0;
      S(tid, RS_FAIL) = ART_SPLIT_CHOLESKY_FAILURE;
    }
    __syncthreads();
    // hard losses: mean squared residual on each side, reduced per (restart,
    // side) in row order
    double sl = 0.0;
    begin_pass();
    for (int64_t c0 = (int64_t)grank * a.CH; c0 < it.n; c0 += (int64_t)gsize * a.CH) {
      const int rows = load_chunk(c0);
      for (int pr = tid; pr < rows * a.Rg; pr += kSplitThreads) {
        const int row = pr / a.Rg, r = pr - row * a.Rg;
        double eL2 = 0.0, eR2 = 0.0;
        if (r < it.rn && S(r, RS_ACTIVE) != 0.0) {
          const double* w = th + r * dt();
          const bool right = right_side(xp + row * xps, w, d, w[d]);
          const double e = ys[row] - fitted((right ? br : bl) + r * a.pmax, row);
          (right ? eR2 : eL2) = e * e;
        }
        cache[row * (2 * a.Rg + 1) + r * 2] = eL2;
        cache[row * (2 * a.Rg + 1) + r * 2 + 1] = eR2;
      }
      __syncthreads();
      if (tid < 2 * it.rn) {
        const int r = tid >> 1, side = tid & 1;
        for (int row = 0; row < rows; ++row) sl += cache[row * (2 * a.Rg + 1) + r * 2 + side];
      }
      __syncthreads();
    }
    if (tid < 2 * it.rn) red[tid] = sl;
    __syncthreads();
    gang_reduce(red, 2 * it.rn);
    if (tid < it.rn && S(tid, RS_ACTIVE) != 0.0) {
      const int r = tid;
      const int nr = (int)S(r, RS_NRIGHT), nl = n - nr;
      const double ll = red[2 * r] / nl, lr = red[2 * r + 1] / nr;
      S(r, RS_HLOSSL) = ll;
      S(r, RS_HLOSSR) = lr;
      S(r, RS_LOSS) = (double)nl / n * ll + (double)nr / n * lr;
    }
    __syncthreads();
  }
  // ----------------------------------------------------------- write results
  if (tid < it.rn && grank == 0) {
    const int r = tid;
    const int64_t kr = (int64_t)k * a.R + it.rbase + r;
    const int dts = a.dmax + 1;
    for (int i = 0; i <= d; ++i) a.r_theta[kr * dts + i] = th[r * dt() + i];
    a.r_fail[kr] = (int)S(r, RS_FAIL);
    a.r_stop[kr] = (int)S(r, RS_STOP);
    a.r_iters[kr] = (int)S(r, RS_ITERS);
    a.r_nright[kr] = (int)S(r, RS_NRIGHT);
    a.r_flags[kr] = (S(r, RS_CONV) != 0.0 ? 1 : 0) | (S(r, RS_FB) != 0.0 ? 2 : 0);
    a.r_fbiter[kr] = (int)S(r, RS_FEASIT);
    a.r_alpha[kr] = P.adaptive_alpha ? S(r, RS_ALPHA) : P.alpha0;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    a.r_loss[kr] = (P.hard_refit && S(r, RS_FAIL) == 0.0) ? S(r, RS_LOSS) : nan;
    a.r_child[kr * 2] = P.hard_refit ? S(r, RS_HLOSSL) : nan;
    a.r_child[kr * 2 + 1] = P.hard_refit ? S(r, RS_HLOSSR) : nan;
    a.r_ridge[kr * 2] = S(r, RS_LAML);
    a.r_ridge[kr * 2 + 1] = S(r, RS_LAMR);
    const bool have = P.hard_refit && S(r, RS_FAIL) == 0.0;
    for (int f = 0; f < it.p; ++f) {
      a.r_beta[(kr * 2) * a.pmax + f] = have ? bl[r * a.pmax + f] : nan;
      a.r_beta[(kr * 2 + 1) * a.pmax + f] = have ? br[r * a.pmax + f] : nan;
    }
  }
  __syncthreads();
  gang_end();
}

// ============================================ warp-per-restart split kernel
// One warp per (node, restart) work item, no block barriers: each warp
// streams its node's rows in tiles of 32, keeps its restart's state in
// registers (uniform across the warp) and a few shared-memory vectors, and
// runs its own projected-gradient loop.  The row products run on the FP64
// tensor path (mma.sync m8n8k4 f64, IEEE FP64 products and sums):
//   * scores and fitted values: [u, f_L, f_R] = psi [w; beta_L; beta_R]
//     (x sits in a contiguous block of psi's columns for every feature kind);
//   * side Grams: G_side += (q_side psi)^T psi, lower-triangular 8 x 8 blocks;
//   * gradient: g = psi^T c over the x columns.
// Gates, losses and Armijo tests are per-row lane work added across the warp.
// The trial step and the next Gram share one pass: the candidate theta_c =
// project(theta + alpha d) is scored as x . w_c - z_c (the frozen-model
// evaluation of objectives.py:131-160), its frozen loss taken at the current
// temperature, and the side Grams at theta_c (at the temperature that
// follows an accepted step) accumulated on the way, so an accepted step
// needs no separate Gram pass.  Same objective, stop rules, Armijo steps,
// AdaptiveAlpha, feasibility tracking, hard partition and refits as the CTA
// kernel above; the summation order differs.

constexpr int kWTile = 32;                                   // rows per tile
constexpr int kWMaxPa = 24;                                  // p + 1 (augmented with y)
constexpr int kWMaxD = 23;                                   // inputs
constexpr int kWThreads = 128;                               // 4 warps per CTA
constexpr int kWGangLog = 12;                                // gang items: n + 1 >= 2^12 rows
constexpr int kWWarps = kWThreads / 32;

// Per-warp shared memory (doubles): psi | cf | sc | tc | th | dn | gr | lf |
// bl | br | A | fidx | xt; psi's row stride is 8 NB + 1 (NB = the kernel's
// block count), the rest follow from (dmax, pmax).
struct WLayout {
  size_t per_warp, total;
  int xs, ps;
};
__host__ __device__ inline WLayout warp_layout(int dmax, int pmax) {
  WLayout L;
  const int pa = pmax + 1, E = pa * (pa + 1) / 2, dt = dmax + 1;
  L.xs = dmax | 1;
  L.ps = (8 * ((pa + 7) / 8)) | 1;
  L.per_warp = (size_t)kWTile * L.ps + 5 * kWTile + 5 * dt + 2 * pmax + E + 2 * pa + pa + kWTile * L.xs;
  L.total = (size_t)kWWarps * L.per_warp * 8;
  return L;
}

// A node of n rows is split by the whole CTA (its warps sharing the tiles)
// when n + 1 >= 2^kWGangLog: on the plan's size buckets, so every gang item
// precedes every other item in the work list.
__device__ __forceinline__ bool warp_gang_item(int64_t n) {
  return ilogb((double)(n + 1)) >= kWGangLog;
}

__device__ __forceinline__ double wbcast_sum(double v) {
  // butterfly sum, then lane 0's value: every lane holds the same bits
  return __shfl_sync(0xffffffffu, warp_sum(v), 0);
}

// first psi column holding x_1 for each feature kind (x is contiguous there)
__device__ __forceinline__ int x_column(int kind) {
  return (kind == ART_FEATURES_POLY1 || kind == ART_FEATURES_POLY2) ? 1 : 0;
}

// NB 8-column blocks of psi (pa <= 8 NB); the score MMAs take NK = 2 NB
// 4-column steps.  Fixed trip counts: padding columns and rows are zeros.
template <int NB>
struct SplitWarp {
  static constexpr int NK = 2 * NB;
  const SplitArgs& a;
  static constexpr int ps = 8 * NB + 1;  // psi row stride (odd, in doubles)
  double* base;                          // this warp's shared-memory region
  bool aff = false;                      // affine features: x is psi's first d columns
  int lane;
  // region pointers, recomputed from the launch's (dmax, pmax) where used
  __device__ double* psi() const { return base; }
  __device__ double* cf() const { return base + kWTile * ps; }
  __device__ double* sc() const { return base + kWTile * ps + 2 * kWTile; }
  __device__ double* tc() const { return base + kWTile * ps + 5 * kWTile; }
  __device__ double* th() const { return tc() + (a.dmax + 1); }
  __device__ double* dn() const { return tc() + 2 * (a.dmax + 1); }
  __device__ double* gr() const { return tc() + 3 * (a.dmax + 1); }
  __device__ double* lf() const { return tc() + 4 * (a.dmax + 1); }
  __device__ double* bl() const { return tc() + 5 * (a.dmax + 1); }
  __device__ double* br() const { return bl() + a.pmax; }
  __device__ double* A() const { return bl() + 2 * a.pmax; }
  __device__ int16_t* fidx() const {
    return (int16_t*)(A() + (a.pmax + 1) * (a.pmax + 2) / 2 + 2 * (a.pmax + 1));
  }
  // the x tile: its own buffer, or for affine features psi itself
  __device__ double* xt() const {
    return aff ? base : (double*)fidx() + (a.pmax + 1);
  }  __device__ int xs() const { return aff ? ps : (a.dmax | 1); }
  __device__ int kq() const { return lane & 3; }   // fragment coordinates of this lane
  __device__ int mq() const { return lane >> 2; }
  // item
  int64_t k, r0, n, xoff, kr;
  int d, kind, p, pa, E, xcol;
  int tail, nks, nbx;  // columns of the last block row; score steps and gradient blocks holding data
  bool narrow;         // tail <= 4: the tail rows of both sides in one MMA per block column
  double ridge, T0;
  // restart state (uniform)
  double loss = 0, dd = 0, tol = 0, gnorm = 0, T = 0, invT = 0, alpha = 0, lamL = 0, lamR = 0;
  double hlossL = 0, hlossR = 0;
  int nright = 0, iters = 0, stop = 0, fail = 0, feasit = -1;
  bool active = false, hasfeas = false, conv = false, fbk = false;

  // gang: the CTA's warps share one large item, warp grank taking tiles
  // grank, grank + gsize, ...; every pass ends with the partial sums of all
  // members added in member order, so each member holds the same totals and
  // runs the same control flow
  int grank = 0, gsize = 1;
  size_t pw;  // doubles per warp region

  __device__ SplitWarp(const SplitArgs& a_, unsigned char* sm, int warp) : a(a_) {
    pw = warp_layout(a.dmax, a.pmax).per_warp;
    base = (double*)sm + (size_t)warp * pw;
    lane = threadIdx.x & 31;
  }
  __device__ int64_t tile0() const { return (int64_t)grank * kWTile; }
  __device__ int64_t tstep() const { return (int64_t)gsize * kWTile; }
  __device__ void gang_bar() const { asm volatile("bar.sync 1, %0;" ::"r"(kWThreads) : "memory"); }
  // Gang sums of per-lane partials: each member stores its partials in
  // slots of its psi region (free between passes), a barrier, then every
  // member adds slot c of all members in member order (gang_end restores
  // psi's zero padding after the second barrier).
  __device__ void gput(int c, double v) const { base[c * kWTile + lane] = v; }
  __device__ double gsum(int c) const {
    const double* b0 = base - (size_t)grank * pw;
    double t = b0[c * kWTile + lane];
    for (int g = 1; g < gsize; ++g) t += b0[(size_t)g * pw + c * kWTile + lane];
    return t;
  }
  __device__ void gang_end() {
    gang_bar();
    for (int f = pa; f < ps; ++f) base[lane * ps + f] = 0.0;
    __syncwarp();
  }

  // Tile rows [t0, t0 + rows): x (coalesced copy) and psi = [phi(x); y],
  // rows past the end zero.  Returns the row count; ends with __syncwarp.
  __device__ int load_tile(int64_t t0, double& yv) {
    const int rows = (int)min((int64_t)kWTile, n - t0);
    const double* src = a.x + xoff + t0 * d;
    const int tot = rows * d;
    const uint32_t inv = 65536u / (uint32_t)d + 1u;  // e / d by a multiply (e < 32 * 23)
    double* xd = xt();
    const int xsv = xs();
    __syncwarp();
    for (int e = lane; e < tot; e += 32) {
      const int rr = (int)(((uint32_t)e * inv) >> 16), i = e - rr * d;
      xd[rr * xsv + i] = __ldg(src + e);
    }
    yv = lane < rows ? __ldg(a.y + r0 + t0 + lane) : 0.0;
    __syncwarp();
    double* pr = psi() + lane * ps;
    const double* xr = xt() + lane * xs();
    if (aff && lane < rows) {
      pr[d] = 1.0;
      pr[p] = yv;
    } else if (lane < rows) {
      for (int f = 0; f < p; ++f) {
        const int ia = fidx()[2 * f], ib = fidx()[2 * f + 1];
        pr[f] = (ia < 0 ? 1.0 : xr[ia]) * (ib < 0 ? 1.0 : xr[ib]);
      }
      pr[p] = yv;
    } else {
      for (int f = 0; f <= p; ++f) pr[f] = 0.0;
    }
    __syncwarp();
    return rows;
  }

  // B fragments of [w; beta_L; beta_R] (columns 0, 1, 2; rows = psi columns)
  // for the score MMAs: lane (k, m) holds B[4 s + k][m] of step s.
  __device__ void score_operand(const double* w, double (&b)[NK]) const {
#pragma unroll
    for (int s = 0; s < NK; ++s) {
      const int f = 4 * s + kq();
      double v = 0.0;
      if (mq() == 0) v = (f >= xcol && f < xcol + d) ? w[f - xcol] : 0.0;
      else if (mq() == 1) v = f < p ? bl()[f] : 0.0;
      else if (mq() == 2) v = f < p ? br()[f] : 0.0;
      b[s] = v;
    }
  }

  // u, f_L, f_R of this lane's row: psi [w; beta_L; beta_R] by MMAs over
  // 8-row blocks, staged through shared memory.  Call after load_tile.
  __device__ void scores(const double (&b)[NK], double& u, double& fl, double& fr) {
#pragma unroll
    for (int rb = 0; rb < 4; ++rb) {
      double c[2] = {0.0, 0.0};
      const double* pr = psi() + (8 * rb + mq()) * ps + kq();
#pragma unroll
      for (int s = 0; s < NK; ++s)
        if (s < NK - 1 || nks == NK) dmma_884(c, pr[4 * s], b[s]);  // the last step may be all padding
      if (kq() == 0) { sc()[8 * rb + mq()] = c[0]; sc()[kWTile + 8 * rb + mq()] = c[1]; }
      else if (kq() == 1) sc()[2 * kWTile + 8 * rb + mq()] = c[0];
    }
    __syncwarp();
    u = sc()[lane];
    fl = sc()[kWTile + lane];
    fr = sc()[2 * kWTile + lane];
    __syncwarp();
  }

  // G_side += (q_side psi)^T psi over the tile (lower 8 x 8 blocks), the
  // weights staged in cf.  Rows past the tile's end are zero rows.
  static constexpr int NBLK = NB * (NB + 1) / 2;  // lower-triangular 8 x 8 blocks
  //
  // Narrow tail (the item's last block row holds tail <= 4 columns, or none):
  // the blocks of the first NB - 1 block rows as above, then the tail rows of
  // both sides in one MMA per block column: A = psi block J, B = [q_L psi_T,
  // q_R psi_T] (columns n < tail: left side, tail <= n < 2 tail: right), so
  // D[m][n] = G_side[T + n'][8 J + m] with T = 8 (NB - 1).  The results sit in
  // cL's last block row; cR's stays zero.
  __device__ void gram_tile(double qL, double qR, double (&cL)[NBLK][2], double (&cR)[NBLK][2]) {
    cf()[lane] = qL;
    cf()[kWTile + lane] = qR;
    __syncwarp();
    if (narrow) {
      constexpr int T = 8 * (NB - 1);
      const int tcol = mq() < tail ? mq() : mq() - tail;
      const bool tl = tail > 0 && mq() < 2 * tail;
#pragma unroll 2
      for (int k0 = 0; k0 < kWTile; k0 += 4) {
        const int row = k0 + kq();
        const double* pr = psi() + row * ps + mq();
        const double ql = cf()[row], qr = cf()[kWTile + row];
        double v[NB];
#pragma unroll
        for (int I = 0; I < NB; ++I) v[I] = pr[8 * I];
#pragma unroll
        for (int I = 0; I < NB - 1; ++I) {
          const double aL = ql * v[I], aR = qr * v[I];
#pragma unroll
          for (int J = 0; J <= I; ++J) {
            dmma_884(cL[I * (I + 1) / 2 + J], aL, v[J]);
            dmma_884(cR[I * (I + 1) / 2 + J], aR, v[J]);
          }
        }
        if (tail > 0) {  // warp-uniform
          const double bt = tl ? (mq() < tail ? ql : qr) * psi()[row * ps + T + tcol] : 0.0;
#pragma unroll
          for (int J = 0; J < NB; ++J) dmma_884(cL[(NB - 1) * NB / 2 + J], v[J], bt);
        }
      }
      __syncwarp();
      return;
    }
#pragma unroll 2
    for (int k0 = 0; k0 < kWTile; k0 += 4) {
      const int row = k0 + kq();
      const double* pr = psi() + row * ps + mq();
      const double ql = cf()[row], qr = cf()[kWTile + row];
      double v[NB];
#pragma unroll
      for (int I = 0; I < NB; ++I) v[I] = pr[8 * I];
#pragma unroll
      for (int I = 0; I < NB; ++I) {
        const double aL = ql * v[I], aR = qr * v[I];
#pragma unroll
        for (int J = 0; J <= I; ++J) {
          dmma_884(cL[I * (I + 1) / 2 + J], aL, v[J]);
          dmma_884(cR[I * (I + 1) / 2 + J], aR, v[J]);
        }
      }
    }
    __syncwarp();
  }

  // g += psi^T c over the tile (column 0 of the MMA output; c staged in cf).
  __device__ void grad_tile(double c, double (&g)[NB][2]) {
    cf()[lane] = c;
    __syncwarp();
#pragma unroll
    for (int k0 = 0; k0 < kWTile; k0 += 4) {
      const int row = k0 + kq();
      const double* pr = psi() + row * ps + mq();
      const double b = mq() == 0 ? cf()[row] : 0.0;
#pragma unroll
      for (int I = 0; I < NB; ++I)
        if (I < NB - 1 || nbx == NB) dmma_884(g[I], pr[8 * I], b);  // blocks holding x columns
    }
    __syncwarp();
  }

  __device__ double gate(double s) const { return a.mixed ? sigm32(s) : sigm(s); }

  __device__ void run(int item);
  // the side Gram blocks (and one extra per-lane partial) summed over the gang
  __device__ void gang_gram(double (&cL)[NBLK][2], double (&cR)[NBLK][2], double* extra = nullptr) {
    static_assert(4 * NBLK + 1 <= ps, "gang slots: 32 x ps doubles of psi");
    if (gsize == 1) return;
#pragma unroll
    for (int q = 0; q < NBLK; ++q) {
      gput(4 * q, cL[q][0]); gput(4 * q + 1, cL[q][1]); gput(4 * q + 2, cR[q][0]); gput(4 * q + 3, cR[q][1]);
    }
    if (extra) gput(4 * NBLK, *extra);
    gang_bar();
#pragma unroll
    for (int q = 0; q < NBLK; ++q) {
      cL[q][0] = gsum(4 * q); cL[q][1] = gsum(4 * q + 1); cR[q][0] = gsum(4 * q + 2); cR[q][1] = gsum(4 * q + 3);
    }
    if (extra) *extra = gsum(4 * NBLK);
    gang_end();
  }
  __device__ bool solve_sides(const double (&cL)[NBLK][2], const double (&cR)[NBLK][2]);
  __device__ void gram_pass(const double* w, bool hard, int req, bool accumulate, double (&cL)[NBLK][2],
                            double (&cR)[NBLK][2]);
  __device__ void resid_pass();
  __device__ double trial_gram_pass(double invT_next, double (&cL)[NBLK][2], double (&cR)[NBLK][2]);
  __device__ void hard_losses();
};

// Both sides' ridge solves from the accumulated Gram blocks; false (restart
// failed) when either factorisation fails.
template <int NB>
__device__ bool SplitWarp<NB>::solve_sides(const double (&cL)[NBLK][2], const double (&cR)[NBLK][2]) {
  double* z_ = A() + E;
  bool ok = true;
  for (int side = 0; side < 2; ++side) {
    __syncwarp();
#pragma unroll
    for (int I = 0; I < NB; ++I)
#pragma unroll
      for (int J = 0; J <= I; ++J)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int i = 8 * I + mq(), j = 8 * J + 2 * kq() + t;
          if ((!narrow || I < NB - 1) && i < pa && j <= i)
            A()[i * (i + 1) / 2 + j] = side ? cR[I * (I + 1) / 2 + J][t] : cL[I * (I + 1) / 2 + J][t];
        }
    if (narrow && tail > 0) {
      // tail rows: lane (m, k) holds D[m][n], n = 2 k + t: side n / tail, row
      // T + n % tail, column 8 J + m
#pragma unroll
      for (int J = 0; J < NB; ++J)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int n_ = 2 * kq() + t;
          if (n_ < 2 * tail && (n_ >= tail) == (side == 1)) {
            const int i = 8 * (NB - 1) + (n_ < tail ? n_ : n_ - tail), j = 8 * J + mq();
            if (i < pa && j <= i) A()[i * (i + 1) / 2 + j] = cL[(NB - 1) * NB / 2 + J][t];
          }
        }
    }
    __syncwarp();
    double lam;
    if (warp_ridge_solve(A(), z_, p, ridge, lam)) {
      ok = false;
      continue;
    }
    double* beta = side ? br() : bl();
    for (int i = lane; i < p; i += 32) beta[i] = z_[i];
    if (side) lamR = lam; else lamL = lam;
  }
  __syncwarp();
  return ok;
}

// Side Grams at theta = (w, w[d]) over all rows.  Soft: gates with the
// weight floor; hard: exact sides (weights 1 / 0) and the right-side count,
// the Gram skipped when a side is below req or `accumulate` is off.
template <int NB>
__device__ void SplitWarp<NB>::gram_pass(const double* w, bool hard, int req, bool accumulate,
                                         double (&cL)[NBLK][2], double (&cR)[NBLK][2]) {
  const double z = w[d];
  double b[NK];
  score_operand(w, b);
#pragma unroll
  for (int q = 0; q < NBLK; ++q) cL[q][0] = cL[q][1] = cR[q][0] = cR[q][1] = 0.0;
  int cnt = 0;
  if (hard) {  // count first: the Grams are needed only when both sides are large enough
    for (int64_t t0 = tile0(); t0 < n; t0 += tstep()) {
      double yv;
      const int rows = load_tile(t0, yv);
      if (lane < rows) cnt += right_side(psi() + lane * ps + xcol, w, d, z) ? 1 : 0;
    }
    if (gsize > 1) {  // integers: exact in any order
      gput(0, (double)cnt);
      gang_bar();
      cnt = (int)gsum(0);
      gang_end();
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    nright = cnt;
    if (nright < req || (int)n - nright < req || !accumulate) return;
  }
  for (int64_t t0 = tile0(); t0 < n; t0 += tstep()) {
    double yv;
    const int rows = load_tile(t0, yv);
    double qL = 0.0, qR = 0.0;
    if (hard) {
      if (lane < rows) {
        const bool right = right_side(psi() + lane * ps + xcol, w, d, z);
        qL = right ? 0.0 : 1.0;
        qR = right ? 1.0 : 0.0;
      }
    } else {
      double u, fl, fr;
      scores(b, u, fl, fr);
      if (lane < rows) {
        const double pi = gate((u - z) * invT);
        qL = fmax(1.0 - pi, a.prm.weight_floor);
        qR = fmax(pi, a.prm.weight_floor);
      }
    }
    gram_tile(qL, qR, cL, cR);
  }
  gang_gram(cL, cR);
}

// Soft residual pass at theta with the current child models: loss,
// gradient, n_right (pi >= 0.5), then the projected gradient, its norm and
// the directional derivative.
template <int NB>
__device__ void SplitWarp<NB>::resid_pass() {
  const double z = th()[d];
  const double inv_n = 1.0 / (double)n;
  double b[NK];
  score_operand(th(), b);
  double g[NB][2];
#pragma unroll
  for (int I = 0; I < NB; ++I) g[I][0] = g[I][1] = 0.0;
  double sl = 0.0, sa = 0.0, snr = 0.0;
  for (int64_t t0 = tile0(); t0 < n; t0 += tstep()) {
    double yv;
    const int rows = load_tile(t0, yv);
    double u, fl, fr;
    scores(b, u, fl, fr);
    double c = 0.0;
    if (lane < rows) {
      const double pi = gate((u - z) * invT);
      const double eL = yv - fl, eR = yv - fr;
      const double eL2 = eL * eL, eR2 = eR * eR;
      c = (eR2 - eL2) * pi * (1.0 - pi) * inv_n;
      sl += (1.0 - pi) * eL2 + pi * eR2;
      sa += c;
      snr += pi >= 0.5 ? 1.0 : 0.0;
    }
    grad_tile(c, g);
  }
  if (gsize > 1) {
#pragma unroll
    for (int I = 0; I < NB; ++I) gput(I, g[I][0]);  // column 0 only is used
    gput(NB, sl); gput(NB + 1, sa); gput(NB + 2, snr);
    gang_bar();
#pragma unroll
    for (int I = 0; I < NB; ++I) g[I][0] = gsum(I);
    sl = gsum(NB); sa = gsum(NB + 1); snr = gsum(NB + 2);
    gang_end();
  }
  // psi column 8 I + m of the gradient sits in lane (k = 0, m), block I
  __syncwarp();
  if (kq() == 0) {
#pragma unroll
    for (int I = 0; I < NB; ++I) {
      const int col = 8 * I + mq() - xcol;
      if (col >= 0 && col < d) gr()[col] = g[I][0] / T;
    }
  }
  const double tot_l = wbcast_sum(sl), tot_a = wbcast_sum(sa), tot_nr = wbcast_sum(snr);
  if (lane == 0) gr()[d] = -tot_a / T;
  __syncwarp();
  loss = tot_l / (double)n;
  nright = (int)tot_nr;
  // projected gradient and its norm (splitters.py:86-98), evaluated by every
  // lane in the same order
  const double* w = th();
  double gw = 0.0, nrm2 = 0.0;
  for (int i = 0; i < d; ++i) gw += gr()[i] * w[i];
  for (int i = 0; i < d; ++i) {
    const double pg = gr()[i] - gw * w[i];
    nrm2 += pg * pg;
  }
  nrm2 += gr()[d] * gr()[d];
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < d; ++i) dn()[i] = -(gr()[i] - gw * w[i]);
    dn()[d] = -gr()[d];
  }
  __syncwarp();
  gnorm = sqrt(nrm2);
  double s = 0.0;
  for (int i = 0; i <= d; ++i) s += gr()[i] * dn()[i];
  dd = s;
}

// One Armijo candidate theta_c (in tc): its frozen-model loss at the current
// temperature (objectives.py:145-156), and the side Grams at theta_c with the
// gates at invT_next, the temperature that follows an accepted step.
template <int NB>
__device__ double SplitWarp<NB>::trial_gram_pass(double invT_next, double (&cL)[NBLK][2], double (&cR)[NBLK][2]) {
  const double z = tc()[d];
  double b[NK];
  score_operand(tc(), b);
#pragma unroll
  for (int q = 0; q < NBLK; ++q) cL[q][0] = cL[q][1] = cR[q][0] = cR[q][1] = 0.0;
  const bool same_t = invT_next == invT;
  double sl = 0.0;
  for (int64_t t0 = tile0(); t0 < n; t0 += tstep()) {
    double yv;
    const int rows = load_tile(t0, yv);
    double u, fl, fr;
    scores(b, u, fl, fr);
    double qL = 0.0, qR = 0.0;
    if (lane < rows) {
      const double pi = gate((u - z) * invT);
      const double eL = yv - fl, eR = yv - fr;
      sl += (1.0 - pi) * (eL * eL) + pi * (eR * eR);
      const double pn = same_t ? pi : gate((u - z) * invT_next);
      qL = fmax(1.0 - pn, a.prm.weight_floor);
      qR = fmax(pn, a.prm.weight_floor);
    }
    gram_tile(qL, qR, cL, cR);
  }
  gang_gram(cL, cR, &sl);
  return wbcast_sum(sl) / (double)n;
}

// Hard losses: mean squared residual of each side's hard model.
template <int NB>
__device__ void SplitWarp<NB>::hard_losses() {
  const double z = th()[d];
  double b[NK];
  score_operand(th(), b);
  double sL = 0.0, sR = 0.0;
  for (int64_t t0 = tile0(); t0 < n; t0 += tstep()) {
    double yv;
    const int rows = load_tile(t0, yv);
    double u, fl, fr;
    scores(b, u, fl, fr);
    if (lane < rows) {
      const bool right = right_side(psi() + lane * ps + xcol, th(), d, z);
      const double e = yv - (right ? fr : fl);
      (right ? sR : sL) += e * e;
    }
  }
  if (gsize > 1) {
    gput(0, sL); gput(1, sR);
    gang_bar();
    sL = gsum(0); sR = gsum(1);
    gang_end();
  }
  const double tl = wbcast_sum(sL), trr = wbcast_sum(sR);
  const int nl = (int)n - nright;
  hlossL = tl / nl;
  hlossR = trr / nright;
  loss = (double)nl / n * hlossL + (double)nright / n * hlossR;
}

template <int NB>
__device__ void SplitWarp<NB>::run(int item) {
  const ArtSplitParams& P = a.prm;
  k = item / a.R;
  kr = (int64_t)item;  // items are k * R + restart
  r0 = a.row_offsets[k];
  n = a.row_offsets[k + 1] - r0;
  xoff = a.x_offsets[k];
  d = a.dims[k];
  kind = a.features[k];
  p = feature_count(d, kind);
  pa = p + 1;
  E = pa * (pa + 1) / 2;
  xcol = x_column(kind);
  tail = pa - 8 * (NB - 1);
  narrow = tail <= 4;
  nks = (p + 3) >> 2;
  nbx = (xcol + d + 7) >> 3;
  T0 = a.temperature[k];
  ridge = a.ridge[k];
  const int req = max(a.min_side ? max(1, a.min_side[k]) : P.min_side_points,
                      (int)ceil(P.min_side_fraction * (double)n));
  const bool fb_allowed = a.fallback ? a.fallback[k] != 0 : false;
  const int M = P.max_iters;
  aff = kind == ART_FEATURES_AFFINE;
  __syncwarp();
  for (int i = lane; i < kWTile * ps; i += 32) psi()[i] = 0.0;  // columns past pa stay zero
  for (int f = lane; f < p; f += 32) {
    int ia, ib;
    feature_factors(d, kind, f, ia, ib);
    fidx()[2 * f] = (int16_t)ia;
    fidx()[2 * f + 1] = (int16_t)ib;
  }
  // initial theta: projected theta0 (splitters.py:379)
  const double* t0 = a.theta0 + kr * a.theta0_stride;
  double nrm2 = 0.0;
  for (int i = 0; i < d; ++i) nrm2 += t0[i] * t0[i];
  const double nrm = sqrt(nrm2);
  active = true;
  fail = 0;
  if (!(nrm > 1e-12) || !isfinite(nrm)) { active = false; fail = ART_SPLIT_INVALID; }
  for (int i = lane; i < d; i += 32) th()[i] = t0[i] / nrm;
  if (lane == 0) th()[d] = t0[d];
  __syncwarp();
  T = T0;
  invT = 1.0 / T0;
  alpha = fmin(fmax(P.alpha0, P.alpha_min), P.alpha_max);
  stop = ART_STOP_MAX_ITERS;
  feasit = -1;
  hasfeas = conv = fbk = false;
  iters = 0;
  nright = 0;
  loss = gnorm = dd = 0.0;
  lamL = lamR = 0.0;
  if (n == 0) { active = false; fail = ART_SPLIT_MIN_SIDE_POINTS; }
  auto record_trace = [&](int iter) {
    if (lane != 0 || grank != 0) return;
    if (a.tr_loss) a.tr_loss[kr * (M + 1) + iter] = loss;
    if (a.tr_gnorm) a.tr_gnorm[kr * (M + 1) + iter] = gnorm;
  };
  auto save_feasible = [&](int it_) {
    if (min(nright, (int)n - nright) >= req) {
      hasfeas = true;
      feasit = it_;
      __syncwarp();
      for (int i = lane; i <= d; i += 32) lf()[i] = th()[i];
      __syncwarp();
    }
  };
  double cL[NBLK][2], cR[NBLK][2];
  // evaluate(theta): child fits from the Grams, then the residual pass
  auto fit_and_resid = [&]() {
    if (!solve_sides(cL, cR)) {
      active = false;
      fail = ART_SPLIT_CHOLESKY_FAILURE;
      return;
    }
    resid_pass();
  };
  if (active) {
    gram_pass(th(), false, 0, true, cL, cR);
    fit_and_resid();
    if (active) {
      tol = P.grad_atol + P.grad_rtol * gnorm;
      save_feasible(0);
      record_trace(0);
    }
  }
  for (int iter = 0; iter < M && active; ++iter) {
    // stop checks (splitters.py:424-437)
    if (gnorm <= tol) { conv = true; stop = ART_STOP_GRADIENT_TOLERANCE; active = false; break; }
    if (dd >= 0.0) { stop = ART_STOP_NON_DESCENT; active = false; break; }
    // temperature after an accepted step (the candidate Grams are taken at it)
    double T_next = T, invT_next = invT;
    if (P.anneal_ratio != 1.0 && P.max_iters > 1) {
      T_next = T0 * pow(P.anneal_ratio, (double)(iter + 1) / (double)(P.max_iters - 1));
      invT_next = 1.0 / T_next;
    }
    // Armijo backtracking, one candidate per pass (optimizers.py:72-121),
    // restarted from the adapted step after a failed attempt
    bool accept = false;
    int failures = 0, nb_ = 0;
    double a_ = P.adaptive_alpha ? alpha : P.alpha0, step = 0.0;
    const int max_trials = (P.max_backtracks + 1) * P.max_line_search_failures;
    for (int trial = 0; trial < max_trials; ++trial) {
      // candidate theta_c = project(theta + alpha d) (splitters.py:451, 497)
      __syncwarp();
      if (lane == 0) {
        double s2 = 0.0;
        for (int i = 0; i < d; ++i) {
          const double v = th()[i] + a_ * dn()[i];
          s2 += v * v;
        }
        const double nw = sqrt(s2);
        for (int i = 0; i < d; ++i) tc()[i] = (th()[i] + a_ * dn()[i]) / nw;
        tc()[d] = th()[d] + a_ * dn()[d];
      }
      __syncwarp();
      const double fv = trial_gram_pass(invT_next, cL, cR);
      const double rhs = __dadd_rn(loss, __dmul_rn(__dmul_rn(P.armijo_c, a_), dd));
      if (fv <= rhs) {
        accept = true;
        step = a_;
        if (P.adaptive_alpha) {  // AdaptiveAlpha.update (optimizers.py:49-66)
          double na;
          if (nb_ == 0) na = step * P.alpha_grow;
          else if (nb_ >= P.heavy_backtrack_threshold) na = step * P.alpha_recovery;
          else na = step / P.rho;
          alpha = fmin(fmax(na, P.alpha_min), P.alpha_max);
        }
        break;
      }
      if (nb_ < P.max_backtracks) {  // next backtrack
        ++nb_;
        a_ *= P.rho;
        continue;
      }
      // attempt failed: the last step tried
      if (P.adaptive_alpha) alpha = fmin(fmax(a_ * P.rho, P.alpha_min), P.alpha_max);
      ++failures;
      int st = -1;
      if (!P.adaptive_alpha) st = ART_STOP_LINE_SEARCH_FAILED;
      else if (failures >= P.max_line_search_failures) st = ART_STOP_MAX_LINE_SEARCH_FAILURES;
      else if (alpha <= P.alpha_min) st = ART_STOP_ALPHA_MIN_REACHED;
      if (st >= 0) {
        stop = st;
        break;
      }
      nb_ = 0;
      a_ = alpha;
    }
    if (!accept) {
      if (stop == ART_STOP_MAX_ITERS) stop = ART_STOP_MAX_LINE_SEARCH_FAILURES;
      active = false;
      break;
    }
    // commit theta <- theta_c, then the new temperature
    __syncwarp();
    for (int i = lane; i <= d; i += 32) th()[i] = tc()[i];
    __syncwarp();
    T = T_next;
    invT = invT_next;
    iters = iter + 1;
    if (lane == 0 && grank == 0) {
      if (a.tr_step) a.tr_step[kr * P.max_iters + iter] = step;
      if (a.tr_back) a.tr_back[kr * P.max_iters + iter] = nb_;
    }
    fit_and_resid();
    if (active) {
      save_feasible(iter + 1);
      record_trace(iter + 1);
    }
  }
  // ------------------------------------------------ finish (splitters.py:584-601)
  if (fail == 0) {
    const bool final_ok = min(nright, (int)n - nright) >= req;
    __syncwarp();
    if (!final_ok && fb_allowed && hasfeas) {
      for (int i = lane; i <= d; i += 32) th()[i] = lf()[i];
      fbk = true;
    }
    __syncwarp();
    double s2 = 0.0;
    for (int i = 0; i < d; ++i) s2 += th()[i] * th()[i];
    const double nw = sqrt(s2);
    __syncwarp();
    if (lane == 0)
      for (int i = 0; i < d; ++i) th()[i] = th()[i] / nw;
    __syncwarp();
    // hard partition: exact sides and right count; hard child fits when asked
    gram_pass(th(), true, req, P.hard_refit != 0, cL, cR);
    if (nright < req || (int)n - nright < req) {
      fail = ART_SPLIT_MIN_SIDE_POINTS;
    } else if (P.hard_refit) {
      if (!solve_sides(cL, cR)) fail = ART_SPLIT_CHOLESKY_FAILURE;
      else hard_losses();
    }
  }
  // ----------------------------------------------------------- write results
  __syncwarp();
  if (lane == 0 && grank == 0) {
    const int dts = a.dmax + 1;
    for (int i = 0; i <= d; ++i) a.r_theta[kr * dts + i] = th()[i];
    a.r_fail[kr] = fail;
    a.r_stop[kr] = stop;
    a.r_iters[kr] = iters;
    a.r_nright[kr] = nright;
    a.r_flags[kr] = (conv ? 1 : 0) | (fbk ? 2 : 0);
    a.r_fbiter[kr] = feasit;
    a.r_alpha[kr] = P.adaptive_alpha ? alpha : P.alpha0;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    const bool have = P.hard_refit && fail == 0;
    a.r_loss[kr] = have ? loss : nan;
    a.r_child[kr * 2] = P.hard_refit ? hlossL : nan;
    a.r_child[kr * 2 + 1] = P.hard_refit ? hlossR : nan;
    a.r_ridge[kr * 2] = lamL;
    a.r_ridge[kr * 2 + 1] = lamR;
    for (int f = 0; f < p; ++f) {
      a.r_beta[(kr * 2) * a.pmax + f] = have ? bl()[f] : nan;
      a.r_beta[(kr * 2 + 1) * a.pmax + f] = have ? br()[f] : nan;
    }
  }
  __syncwarp();
}

// Resident 4-warp CTAs per SM: 4 (16 warps, a 128-register cap) for up to
// two blocks; 3 (12 warps, 168 registers) for three, whose six Gram blocks
// per side would spill under the tighter cap.
template <int NB>
__global__ void __launch_bounds__(kWThreads, NB == 3 ? 3 : 4) split_warp_kernel(SplitArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_q;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SplitWarp<NB> W(a, smem, warp);
  const int count = a.counts[0];
  // Items come largest first.  While they are large the whole CTA takes one
  // at a time (a gang of all its warps); from the first small item on, each
  // warp pops its own, warp 0 starting with the CTA's last pop.  (One call
  // site of run keeps it inlined and the state in registers.)
  bool cta_phase = true;
  for (;;) {
    int item = -1;
    if (cta_phase) {
      if (threadIdx.x == 0) s_q = atomicAdd(&a.counts[1], 1);
      __syncthreads();
      const int q = s_q;
      __syncthreads();
      if (q >= count) return;
      item = a.items[q].x;
      const int64_t k = item / a.R;
      if (warp_gang_item(a.row_offsets[k + 1] - a.row_offsets[k])) {
        W.grank = warp;
        W.gsize = kWWarps;
      } else {
        cta_phase = false;
        W.grank = 0;
        W.gsize = 1;
        if (warp != 0) item = -1;
      }
    }
    if (item < 0) {
      int q = 0;
      if (lane == 0) q = atomicAdd(&a.counts[1], 1);
      q = __shfl_sync(0xffffffffu, q, 0);
      if (q >= count) return;
      item = a.items[q].x;
    }
    W.run(item);
  }
}

// MINB resident CTAs per SM: 1 keeps every register a thread wants and the
// deepest row ring; 2 doubles the warps that hide the per-row latency of the
// passes at the cost of a 128-register cap and half the shared memory
template <int TC, int MINB, int TCG = 0>
__global__ void __launch_bounds__(kSplitThreads, MINB) split_kernel(SplitArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item;
  SplitCta<TC, TCG> cta(a, smem);
  __shared__ uint32_t s_tmem;
  if (threadIdx.x == 0) {
    for (int i = 0; i < a.S; ++i) mbar_init(&cta.rbar[i], 1);
    if constexpr (TCG) mbar_init((uint64_t*)(smem + cta.L.tcbar), 1);
    fence_mbar_init();
  }
  if constexpr (TCG) {
    if ((threadIdx.x >> 5) == 0) {
      tmem_alloc(&s_tmem, kTcCols);
      tmem_relinquish();
    }
    tc_fence_before();
  }
  __syncthreads();
  if constexpr (TCG) {
    tc_fence_after();
    cta.tmem = s_tmem;
  }
  const int count = a.counts[0];
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&a.counts[1], 1);
    __syncthreads();
    const int q = s_item;
    __syncthreads();
    if (q >= count) break;
    const int4 e = a.items[q];
    cta.run(e.x, e.y, e.z);
  }
  cta.ring_drain();
  if constexpr (TCG) {  // release TMEM after a bounded wait for this CTA's MMAs
    cta.tc_wait_all();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(cta.tmem, kTcCols);
  }
}

// Per node: best non-fallback restart by hard loss, else best fallback,
// else the last failure (splitters.py:354-363); copy it to the outputs.
__global__ void split_select(SplitArgs a, ArtSplitResult out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.K) return;
  const int d = a.dims[k], p = feature_count(d, a.features[k]);
  int best = -1, best_fb = -1, last_fail = -1;
  for (int r = 0; r < a.R; ++r) {
    const int64_t kr = k * a.R + r;
    if (a.r_fail[kr] != 0) { last_fail = r; continue; }
    const bool fb = (a.r_flags[kr] & 2) != 0;
    const double l = a.r_loss[kr];
    if (!a.prm.hard_refit) { if (best < 0) best = r; continue; }
    if (fb) { if (best_fb < 0 || l < a.r_loss[k * a.R + best_fb]) best_fb = r; }
    else if (best < 0 || l < a.r_loss[k * a.R + best]) best = r;
  }
  int pick = best >= 0 ? best : (best_fb >= 0 ? best_fb : last_fail);
  if (pick < 0) pick = 0;
  const int64_t kr = k * a.R + pick;
  const int dts = a.dmax + 1;
  for (int i = 0; i <= d; ++i) out.theta[k * out.theta_stride + i] = a.r_theta[kr * dts + i];
  if (out.beta)
    for (int f = 0; f < p; ++f) {
      out.beta[(k * 2) * out.beta_stride + f] = a.r_beta[(kr * 2) * a.pmax + f];
      out.beta[(k * 2 + 1) * out.beta_stride + f] = a.r_beta[(kr * 2 + 1) * a.pmax + f];
    }
  if (out.loss) out.loss[k] = a.r_loss[kr];
  if (out.child_loss) { out.child_loss[2 * k] = a.r_child[2 * kr]; out.child_loss[2 * k + 1] = a.r_child[2 * kr + 1]; }
  if (out.ridge_effective) { out.ridge_effective[2 * k] = a.r_ridge[2 * kr]; out.ridge_effective[2 * k + 1] = a.r_ridge[2 * kr + 1]; }
  if (out.n_right) out.n_right[k] = a.r_nright[kr];
  if (out.n_iters) out.n_iters[k] = a.r_iters[kr];
  if (out.stop_reason) out.stop_reason[k] = a.r_stop[kr];
  // a bounded row-copy wait gave up somewhere in the level: no result is trusted
  const bool lost = a.counts[kErrSlot] != 0;
  if (out.failure) out.failure[k] = lost ? ART_SPLIT_INVALID : ((best >= 0 || best_fb >= 0) ? 0 : a.r_fail[kr]);
  if (out.flags) out.flags[k] = a.r_flags[kr] | (pick << 8);
  if (out.fallback_iteration) out.fallback_iteration[k] = a.r_fbiter[kr];
  if (out.final_alpha) out.final_alpha[k] = a.r_alpha[kr];
}

// Device initialisation of theta0 when none is supplied: w ~ N(0, I) from
// Philox keyed by (seed, node, restart), normalised; z = median(X w) by
// selection (numpy's median: mean of the two middle values for even n).
__global__ void split_init_theta(SplitArgs a, double* theta0, int64_t stride) {
  const int64_t kr = blockIdx.x;
  if (kr >= a.K * a.R) return;
  const int64_t k = kr / a.R;
  const int d = a.dims[k];
  const int64_t r0 = a.row_offsets[k], n = a.row_offsets[k + 1] - r0;
  const int64_t xoff = a.x_offsets[k];
  __shared__ double w[ART_MAX_DIM + 1];
  if (threadIdx.x == 0) {
    double nrm2 = 0.0;
    // counter: (node k, restart) or, with per-node keys, (restart, node key):
    // the latter does not depend on the node's position in the batch
    const int64_t rr = kr - k * a.R;
    const uint64_t nk = a.node_keys ? a.node_keys[k] : 0ull;
    for (int i = 0; i < d; i += 2) {
      Philox4 r = a.node_keys
                      ? philox4x32_10((uint32_t)rr, (uint32_t)nk, (uint32_t)i, (uint32_t)(nk >> 32) ^ 0x5eed0000u,
                                      (uint32_t)a.prm.seed, (uint32_t)(a.prm.seed >> 32))
                      : philox4x32_10((uint32_t)kr, (uint32_t)(kr >> 32), (uint32_t)i, 0x5eedu,
                                      (uint32_t)a.prm.seed, (uint32_t)(a.prm.seed >> 32));
      double z0, z1;
      normal_pair(r, z0, z1);
      w[i] = z0;
      if (i + 1 < d) w[i + 1] = z1;
    }
    for (int i = 0; i < d; ++i) nrm2 += w[i] * w[i];
    double nrm = sqrt(nrm2);
    if (nrm <= 1e-12) { w[0] = 1.0; for (int i = 1; i < d; ++i) w[i] = 0.0; nrm = 1.0; }
    for (int i = 0; i < d; ++i) w[i] /= nrm;
  }
  __syncthreads();
  // median of u = X w by a radix select on the order-preserving 64-bit image
  // of the doubles (sign bit flipped for positives, all bits flipped for
  // negatives): six digit passes of up to 11 bits narrow a prefix to the
  // exact key of the m-th smallest u, each pass recomputing u and counting
  // the rows that share the prefix into a shared histogram.
  constexpr int kBins = 2048;
  __shared__ unsigned int hist[kBins];
  __shared__ unsigned long long s_pre;
  __shared__ long long s_m;
  auto ukey = [](double v) -> unsigned long long {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
  };
  auto from_ukey = [](unsigned long long k) -> double {
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
  };
  auto u_of = [&](int64_t i) {
    double u = 0.0;
    for (int cc = 0; cc < d; ++cc) u = fma(a.x[xoff + i * d + cc], w[cc], u);
    return u;
  };
  auto kth = [&](long long m) -> unsigned long long {
    unsigned long long prefix = 0ull, mask = 0ull;
    // digits (shift, width): bits 53..63, 42..52, 31..41, 20..30, 9..19, 0..8
    for (int pass = 0; pass < 6; ++pass) {
      const int sh = pass < 5 ? 53 - 11 * pass : 0;
      const int width = pass < 5 ? 11 : 9;
      const unsigned long long dmask = (1ull << width) - 1ull;
      for (int b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0u;
      __syncthreads();
      for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long k = ukey(u_of(i));
        if ((k & mask) == prefix) atomicAdd(&hist[(k >> sh) & dmask], 1u);
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        // warp 0: lane l sums bins [64 l, 64 l + 64); an exclusive scan over
        // the lanes finds the lane holding rank m, which scans its own bins
        const int l = threadIdx.x;
        long long part = 0;
        for (int b = 64 * l; b < 64 * l + 64; ++b) part += hist[b];
        long long incl = part;
        for (int o = 1; o < 32; o <<= 1) {
          const long long t = __shfl_up_sync(0xffffffffu, incl, o);
          if (l >= o) incl += t;
        }
        const long long excl = incl - part;
        const unsigned hit = __ballot_sync(0xffffffffu, m >= excl && m < incl);
        const int owner = hit ? __ffs(hit) - 1 : 31;
        if (l == owner) {
          long long mm = m - excl;
          int b = 64 * l;
          for (; b < 64 * l + 63; ++b) {
            if (mm < (long long)hist[b]) break;
            mm -= hist[b];
          }
          s_pre = prefix | ((unsigned long long)b << sh);
          s_m = mm;
        }
      }
      __syncthreads();
      prefix = s_pre;
      m = s_m;
      mask |= dmask << sh;
      __syncthreads();
    }
    return prefix;
  };
  if (n == 0) {
    if (threadIdx.x == 0) { for (int i = 0; i < d; ++i) theta0[kr * stride + i] = w[i]; theta0[kr * stride + d] = 0.0; }
    return;
  }
  const unsigned long long k1 = kth((n - 1) / 2);
  const double v1 = from_ukey(k1);
  double v2 = v1;
  if (n % 2 == 0) {
    // the next order statistic: v1 again if more than n/2 keys are <= k1,
    // else the smallest u above v1
    __shared__ unsigned long long s_min;
    __shared__ long long s_cnt;
    if (threadIdx.x == 0) { s_min = ~0ull; s_cnt = 0; }
    __syncthreads();
    long long cnt = 0;
    unsigned long long mn = ~0ull;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      const unsigned long long k = ukey(u_of(i));
      if (k <= k1) ++cnt;
      else if (k < mn) mn = k;
    }
    atomicAdd((unsigned long long*)&s_cnt, (unsigned long long)cnt);
    atomicMin(&s_min, mn);
    __syncthreads();
    v2 = s_cnt > n / 2 ? v1 : from_ukey(s_min);
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < d; ++i) theta0[kr * stride + i] = w[i];
    theta0[kr * stride + d] = (n % 2 == 0) ? 0.5 * (v1 + v2) : v1;
  }
}

struct SplitWs {
  size_t counts, items, gang_rec, slot_flags, gang_scratch, theta0, r_theta, r_loss, r_beta, r_child,
      r_ridge, r_i, r_alpha, total;
  int nslots, gang_P;
  bool gang_on;
};
// Gangs run only for levels with at most two restarts per node (one or two
// work items per node), where a large node would otherwise hold one SM for
// the whole level.
SplitWs split_ws(int64_t K, int R, int dmax, int pmax) {
  SplitWs w;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = (o + bytes + 255) & ~(size_t)255; return at; };
  w.gang_on = R <= 2;
  const int pa = pmax + 1, E = pa * (pa + 1) / 2;
  w.gang_P = w.gang_on ? std::max(std::max(E * 4, 2 * (dmax + 3)), 256) : 0;
  w.nslots = w.gang_on ? device_sm_count() + 2 : 0;
  w.counts = take(4 * (kErrSlot + 1));
  w.items = take(16 * (size_t)K * R * (w.gang_on ? kGangMax : 1));
  w.gang_rec = take(16 * (size_t)K * R);
  w.slot_flags = take(4 * (size_t)std::max(w.nslots, 1));
  w.gang_scratch = take(8 * (size_t)w.nslots * 2 * kGangMax * w.gang_P);
  w.theta0 = take(8 * (size_t)K * R * (ART_MAX_DIM + 1));
  w.r_theta = take(8 * (size_t)K * R * (dmax + 1));
  w.r_loss = take(8 * (size_t)K * R);
  w.r_beta = take(8 * (size_t)K * R * 2 * pmax);
  w.r_child = take(8 * (size_t)K * R * 2);
  w.r_ridge = take(8 * (size_t)K * R * 2);
  w.r_i = take(4 * (size_t)K * R * 6);
  w.r_alpha = take(8 * (size_t)K * R);
  w.total = o;
  return w;
}

int choose_rg(int R, int pa, int cap, int& TC) {
  // largest group (<= 16 restarts, <= cap when cap > 0) whose Gram tiles fit
  // 256 threads and the accumulators a modest shared-memory budget
  const int E = pa * (pa + 1) / 2;
  const int top = std::min(std::min(R, kMaxRg), cap > 0 ? cap : kMaxRg);
  for (int rg = top; rg >= 1; --rg) {
    const int c2 = 2 * rg;
    const int tc = c2 >= 8 ? 8 : (c2 >= 4 ? 4 : 2);
    const int te = 32 / tc;
    const int tiles = ((E + te - 1) / te) * ((c2 + tc - 1) / tc);
    if (tiles <= kSplitThreads && (size_t)E * c2 * 8 <= 64 * 1024) { TC = tc; return rg; }
  }
  TC = 2;
  return 0;
}

}  // namespace
}  // namespace art

using namespace art;

extern "C" size_t art_split_workspace_size(int64_t count, int32_t n_restarts, int32_t max_dim,
                                           int32_t max_features) {
  if (count < 0 || n_restarts < 1) return 0;
  return split_ws(count, n_restarts, std::max(max_dim, 1), std::max(max_features, 1)).total;
}

extern "C" int art_split_level(const ArtSplitProblem* pr, const ArtSplitParams* prm,
                               const ArtSplitResult* out, void* workspace, size_t ws_bytes,
                               art_stream_t stream) {
  cudaGetLastError();
  if (!pr || !prm || !out) { set_error("art_split_level: null argument"); return ART_E_INVALID; }
  const int64_t K = pr->seg.count;
  if (K < 0) { set_error("art_split_level: negative count"); return ART_E_INVALID; }
  if (K == 0) return ART_OK;
  if (!pr->seg.row_offsets || !pr->seg.x_offsets || !pr->seg.dims || !pr->seg.features || !pr->x ||
      !pr->y || !pr->temperature || !pr->ridge || !out->theta) {
    set_error("art_split_level: null device pointer");
    return ART_E_INVALID;
  }
  if (pr->max_dim < 1 || pr->max_dim > ART_MAX_DIM || pr->max_features < 1 || pr->max_features > kMaxP) {
    set_error("art_split_level: max_dim in [1, %d] and max_features in [1, %d] required", ART_MAX_DIM, kMaxP);
    return ART_E_UNSUPPORTED;
  }
  if (prm->n_restarts < 1 || prm->max_iters < 0 || prm->max_backtracks < 0 ||
      prm->max_line_search_failures < 1 || !(prm->rho > 0.0 && prm->rho < 1.0) ||
      !(prm->armijo_c > 0.0 && prm->armijo_c < 1.0) || !(prm->alpha0 > 0.0) ||
      !(prm->alpha_min > 0.0) || prm->alpha_max < prm->alpha_min || prm->min_side_points < 1 ||
      !(prm->min_side_fraction >= 0.0 && prm->min_side_fraction < 0.5) || !(prm->anneal_ratio > 0.0) ||
      prm->group_restarts < 0 || prm->trial_steps < 0 || prm->ctas_per_sm < 0 || prm->ctas_per_sm > 2 ||
      prm->tensor_gram < 0 || prm->tensor_gram > 1 || prm->restart_warps < 0 || prm->restart_warps > 1) {
    set_error("art_split_level: invalid splitter parameters");
    return ART_E_INVALID;
  }
  if (prm->precision != ART_PRECISION_FP64 && prm->precision != ART_PRECISION_MIXED) {
    set_error("art_split_level: precision must be ART_PRECISION_FP64 or ART_PRECISION_MIXED");
    return ART_E_INVALID;
  }
  if (out->theta_stride < pr->max_dim + 1 || (out->beta && out->beta_stride < pr->max_features)) {
    set_error("art_split_level: output strides too small");
    return ART_E_INVALID;
  }
  const int R = prm->n_restarts;
  int TC = 2;
  int Rg = choose_rg(R, pr->max_features + 1, prm->group_restarts, TC);
  if (Rg < 1) { set_error("art_split_level: model too large for the split kernel"); return ART_E_UNSUPPORTED; }
  // Mixed form with tensor_gram: the soft-pass Grams go to the tensor cores
  // when the entries fit two M = 128 tiles and the operands fit shared
  // memory next to the rest (one CTA per SM); the restarts of a work item
  // share one operand generation per chunk.
  int use_tc = 0;
  {
    const int pa = pr->max_features + 1, E = pa * (pa + 1) / 2;
    if (prm->precision == ART_PRECISION_MIXED && prm->tensor_gram && E <= kTcEntries) {
      int tc_cols = 2;
      const int rg = choose_rg(R, pa, prm->group_restarts, tc_cols);
      const int H = std::min(std::min(prm->trial_steps > 0 ? prm->trial_steps : 4, std::max(1, kSplitThreads / std::max(rg, 1))),
                             prm->max_backtracks + 1);
      if (rg >= 1 && split_layout(pr->max_dim, pr->max_features, rg, H, 2, kTcRows, 1).total <= 227 * 1024) {
        use_tc = 1;
        Rg = rg;
        TC = tc_cols;
      }
    }
  }
  // Warp-per-restart form: asked for, the level fits its register tiles and
  // no tensor-core Gram is in use
  const bool use_warp = prm->restart_warps == 1 && !use_tc && pr->max_dim <= kWMaxD &&
                        pr->max_features + 1 <= kWMaxPa;
  const SplitWs wl = split_ws(K, R, pr->max_dim, pr->max_features);
  if (!workspace || ws_bytes < wl.total) {
    set_error("art_split_level: workspace %zu bytes < required %zu", ws_bytes, wl.total);
    return ART_E_WORKSPACE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* ws = (unsigned char*)workspace;
  SplitArgs a{};
  a.K = K;
  a.row_offsets = pr->seg.row_offsets; a.x_offsets = pr->seg.x_offsets;
  a.dims = pr->seg.dims; a.features = pr->seg.features;
  a.x = pr->x; a.y = pr->y; a.temperature = pr->temperature; a.ridge = pr->ridge;
  a.parent_loss = pr->parent_loss; a.fallback = pr->min_side_fallback;
  a.node_keys = pr->node_keys;
  a.min_side = pr->min_side_points;
  a.prm = *prm;
  a.R = R; a.Rg = Rg; a.groups = (R + Rg - 1) / Rg;
  a.dmax = pr->max_dim; a.pmax = pr->max_features; a.TC = TC;
  a.mixed = prm->precision == ART_PRECISION_MIXED ? 1 : 0;
  a.tc = use_tc;
  // default: four speculative Armijo steps per trial pass (adaptive step
  // sizes are usually accepted within the first two; longer backtracks take
  // further passes), spare threads share the rows instead
  a.H = std::min(4, std::max(1, kSplitThreads / Rg));
  if (prm->trial_steps > 0) a.H = std::min(prm->trial_steps, std::max(1, kSplitThreads / Rg));
  a.H = std::min(a.H, prm->max_backtracks + 1);
  a.r_theta = (double*)(ws + wl.r_theta); a.r_loss = (double*)(ws + wl.r_loss);
  a.r_beta = (double*)(ws + wl.r_beta); a.r_child = (double*)(ws + wl.r_child);
  a.r_ridge = (double*)(ws + wl.r_ridge);
  int32_t* ri = (int32_t*)(ws + wl.r_i);
  a.r_nright = ri; a.r_iters = ri + K * R; a.r_stop = ri + 2 * K * R; a.r_fail = ri + 3 * K * R;
  a.r_flags = ri + 4 * K * R; a.r_fbiter = ri + 5 * K * R;
  a.r_alpha = (double*)(ws + wl.r_alpha);
  a.tr_loss = out->trace_loss; a.tr_step = out->trace_step; a.tr_back = out->trace_backtracks;
  a.tr_gnorm = out->trace_grad_norm;
  a.counts = (int32_t*)(ws + wl.counts); a.items = (int4*)(ws + wl.items);
  a.gang_on = wl.gang_on && a.Rg <= 2 ? 1 : 0;
  a.nslots = wl.nslots;
  a.gang_P = wl.gang_P;
  a.gang_rec = (int4*)(ws + wl.gang_rec);
  a.slot_flags = (int32_t*)(ws + wl.slot_flags);
  a.gang_scratch = (double*)(ws + wl.gang_scratch);
  if (pr->theta0) {
    a.theta0 = pr->theta0;
    a.theta0_stride = pr->theta_stride;
  } else {
    a.theta0 = (double*)(ws + wl.theta0);
    a.theta0_stride = ART_MAX_DIM + 1;
    prof_begin("split_init_theta", s);
    split_init_theta<<<(unsigned)(K * R), 256, 0, s>>>(a, (double*)(ws + wl.theta0), ART_MAX_DIM + 1);
    prof_end(s);
    count_launch();
  }
  // CTA form without the tensor-core Gram, one or two restarts per CTA: side
  // Grams as FP64 MMA tiles when the (side, block) items fit the warps'
  // accumulators (measured on the B200: 1.8x on wide single-restart levels;
  // with 4 restarts per CTA the thread-tile sums are faster)
  if (!use_warp && !use_tc && Rg <= 2) {
    const int nb = (pr->max_features + 1 + 7) / 8;
    a.dg = 2 * Rg * (nb * (nb + 1) / 2) <= kWarps * kDgMax ? 1 : 0;
  }
  if (use_warp) {
    // one work item per (node, restart), largest nodes first
    a.Rg = 1;
    a.groups = R;
    a.TC = 2;
    a.H = 1;
    a.gang_on = 0;
  }
  if (cudaMemsetAsync(a.counts, 0, 4 * (kErrSlot + 1), s) != cudaSuccess) return check_launch("memset");
  if (a.gang_on &&
      (cudaMemsetAsync(a.gang_rec, 0, 16 * (size_t)K * a.groups, s) != cudaSuccess ||
       cudaMemsetAsync(a.slot_flags, 0, 4 * (size_t)std::max(a.nslots, 1), s) != cudaSuccess))
    return check_launch("memset");
  const unsigned pg = (unsigned)((K * a.groups + 255) / 256);
  prof_begin("split_plan", s);
  split_plan_hist<<<pg, 256, 0, s>>>(a);
  split_plan_scan<<<1, 32, 0, s>>>(a);
  split_plan_scatter<<<pg, 256, 0, s>>>(a);
  prof_end(s);
  count_launch(); count_launch(); count_launch();
  if (use_warp) {
    const size_t wsm = warp_layout(a.dmax, a.pmax).total;
    auto launch_warp = [&](auto kern) -> int {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm) != cudaSuccess) {
        cudaGetLastError();
        set_error("art_split_level: cannot reserve %zu bytes of shared memory", wsm);
        return ART_E_UNSUPPORTED;
      }
      const int occ = resident_ctas((const void*)kern, kWThreads, wsm);
      const int64_t resident = (int64_t)device_sm_count() * std::max(occ, 1);
      const int64_t grid = std::min<int64_t>(resident, (K * R + kWWarps - 1) / kWWarps);
      prof_begin("split_level", s);
      kern<<<(unsigned)std::max<int64_t>(grid, 1), kWThreads, wsm, s>>>(a);
      prof_end(s);
      count_launch();
      return check_launch("split_level");
    };
    const int nbk = (a.pmax + 1 + 7) / 8;  // 8-column blocks of the widest psi
    int rcw;
    if (nbk == 1) rcw = launch_warp(split_warp_kernel<1>);
    else if (nbk == 2) rcw = launch_warp(split_warp_kernel<2>);
    else rcw = launch_warp(split_warp_kernel<3>);
    if (rcw) return rcw;
    prof_begin("split_select", s);
    split_select<<<(unsigned)((K + 127) / 128), 128, 0, s>>>(a, *out);
    prof_end(s);
    count_launch();
    return check_launch("split_select");
  }
  // longest chunk (fewer block barriers per row) with a ring of at least 4
  // stages (2 at two CTAs per SM) that fits shared memory, then the deepest
  // ring for that chunk; two CTAs per SM fall back to one when even the
  // shortest chunk does not fit half the SM's shared memory
  int minb = prm->ctas_per_sm == 2 ? 2 : 1;
  if (a.tc) {
    // one CTA per SM: chunks of kTcRows rows and the deepest ring that fits
    minb = 1;
    a.CH = 128;
    while (a.CH > kTcRows && split_layout(a.dmax, a.pmax, a.Rg, a.H, 2, a.CH, 1).total > 227 * 1024) a.CH >>= 1;
    a.S = kMaxStages;
    while (a.S > 2 && split_layout(a.dmax, a.pmax, a.Rg, a.H, a.S, a.CH, 1).total > 227 * 1024) --a.S;
  } else {
    if (minb == 2 && split_layout(a.dmax, a.pmax, a.Rg, a.H, 1, 32, 0, a.dg).total > kHalfSmem) minb = 1;
    const size_t chunk_budget = minb == 2 ? 100 * 1024 : 200 * 1024;
    const size_t smem_budget = minb == 2 ? kHalfSmem : 227 * 1024;
    const int min_stages = minb == 2 ? 2 : 4;
    a.CH = kMaxCH;
    while (a.CH > 32 && split_layout(a.dmax, a.pmax, a.Rg, a.H, min_stages, a.CH, 0, a.dg).total > chunk_budget)
      a.CH >>= 1;
    a.S = kMaxStages;
    while (a.S > 1 && split_layout(a.dmax, a.pmax, a.Rg, a.H, a.S, a.CH, 0, a.dg).total > smem_budget) --a.S;
  }
  const size_t smem = split_layout(a.dmax, a.pmax, a.Rg, a.H, a.S, a.CH, a.tc, a.dg).total;
  if (smem > 227 * 1024) { set_error("art_split_level: shared memory %zu too large", smem); return ART_E_UNSUPPORTED; }
  auto launch = [&](auto kern) -> int {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      set_error("art_split_level: cannot reserve %zu bytes of shared memory", smem);
      return ART_E_UNSUPPORTED;
    }
    const int occ = resident_ctas((const void*)kern, kSplitThreads, smem);
    // with gangs every resident CTA may be needed (a gang's members must all
    // be resident), so the grid is the full residency
    const int64_t resident = (int64_t)device_sm_count() * std::max(occ, 1);
    const int64_t grid = a.gang_on ? resident : std::min<int64_t>(resident, K * a.groups);
    prof_begin("split_level", s);
    kern<<<(unsigned)std::max<int64_t>(grid, 1), kSplitThreads, smem, s>>>(a);
    prof_end(s);
    count_launch();
    return check_launch("split_level");
  };
  int rc;
  if (a.tc) {
    if (TC == 8) rc = launch(split_kernel<8, 1, 1>);
    else if (TC == 4) rc = launch(split_kernel<4, 1, 1>);
    else rc = launch(split_kernel<2, 1, 1>);
  } else if (minb == 2) {
    if (TC == 8) rc = launch(split_kernel<8, 2>);
    else if (TC == 4) rc = launch(split_kernel<4, 2>);
    else rc = launch(split_kernel<2, 2>);
  } else {
    if (TC == 8) rc = launch(split_kernel<8, 1>);
    else if (TC == 4) rc = launch(split_kernel<4, 1>);
    else rc = launch(split_kernel<2, 1>);
  }
  if (rc) return rc;
  prof_begin("split_select", s);
  split_select<<<(unsigned)((K + 127) / 128), 128, 0, s>>>(a, *out);
  prof_end(s);
  count_launch();
  return check_launch("split_select");
}
