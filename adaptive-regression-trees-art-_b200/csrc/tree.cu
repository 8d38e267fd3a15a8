// tree.cu -- node-sorted stable partition of rows by a split plane, and
// batched tree routing + leaf prediction.
//
// Routing rule everywhere: w . x - z >= 0 goes right (builder.py:494,
// tree.py:159, splitters.py:618).  The side is the sign of the exact value
// of w . x - z (right_side: a compensated dot product, and exact expansion
// arithmetic for the rare scores within its error bound); numpy's own
// rounded X @ w - z can disagree only where its rounding error exceeds
// |w . x - z|.
#include "common.cuh"

namespace art {
namespace {

constexpr int kPartThreads = 256;

__global__ void __launch_bounds__(kPartThreads)
    partition_kernel(ArtSegments seg, const double* x, const double* theta, int64_t ts,
                     const int8_t* split, int64_t* perm, int32_t* n_right) {
  const int k = blockIdx.x;
  const int64_t r0 = seg.row_offsets[k], n = seg.row_offsets[k + 1] - r0;
  const int64_t xoff = seg.x_offsets[k];
  const int d = seg.dims[k];
  const bool do_split = split == nullptr || split[k] != 0;
  __shared__ double w[ART_MAX_DIM + 1];
  __shared__ int64_t s_base_left, s_base_right;
  __shared__ int warp_tot[kPartThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i <= d; i += kPartThreads) w[i] = theta[(int64_t)k * ts + i];
  __syncthreads();
  // pass 1: count right rows
  int local = 0;
  if (do_split)
    for (int64_t r = tid; r < n; r += kPartThreads) {
      local += right_side(x + xoff + r * d, w, d, w[d]) ? 1 : 0;
    }
  int tot = warp_sum(local);
  if (lane == 0) warp_tot[warp] = tot;
  __syncthreads();
  if (tid == 0) {
    int64_t t = 0;
    for (int i = 0; i < kPartThreads / 32; ++i) t += warp_tot[i];
    s_base_left = 0;
    s_base_right = n - t;
    if (n_right) n_right[k] = (int32_t)t;
  }
  __syncthreads();
  // pass 2: stable scatter in tiles of kPartThreads rows
  for (int64_t base = 0; base < n; base += kPartThreads) {
    const int64_t r = base + tid;
    int right = 0;
    if (r < n && do_split) right = right_side(x + xoff + r * d, w, d, w[d]) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, right);
    const unsigned inb = __ballot_sync(0xffffffffu, r < n);
    const int wr = __popc(bal), wl = __popc(inb & ~bal);
    __shared__ int s_wr[kPartThreads / 32], s_wl[kPartThreads / 32];
    if (lane == 0) { s_wr[warp] = wr; s_wl[warp] = wl; }
    __syncthreads();
    int pre_r = 0, pre_l = 0, tile_r = 0, tile_l = 0;
    for (int i = 0; i < kPartThreads / 32; ++i) {
      if (i < warp) { pre_r += s_wr[i]; pre_l += s_wl[i]; }
      tile_r += s_wr[i];
      tile_l += s_wl[i];
    }
    const unsigned lt = (1u << lane) - 1u;
    if (r < n) {
      int64_t pos;
      if (right) pos = s_base_right + pre_r + __popc(bal & lt);
      else pos = s_base_left + pre_l + __popc(inb & ~bal & lt);
      perm[r0 + pos] = r0 + r;
    }
    __syncthreads();
    if (tid == 0) { s_base_right += tile_r; s_base_left += tile_l; }
    __syncthreads();
  }
}

__device__ inline double leaf_predict(const double* xr, int d, int kind, const double* c) {
  const int p = feature_count(d, kind);
  double s = 0.0;
  for (int f = 0; f < p; ++f) {
    int a, b;
    feature_factors(d, kind, f, a, b);
    const double v = (a < 0 ? 1.0 : xr[a]) * (b < 0 ? 1.0 : xr[b]);
    s = fma(v, c[f], s);
  }
  return s;
}

__global__ void predict_kernel(int d, int64_t n_nodes, const int32_t* child, const double* theta,
                               int64_t ts, const double* coef, int64_t cs, const int32_t* features,
                               int64_t n, const double* x, int32_t* leaf, double* pred) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* xr = x + i * d;
  int node = 0;
  for (int64_t guard = 0; guard < n_nodes && child[2 * node] >= 0; ++guard) {
    const double* t = theta + (int64_t)node * ts;
    node = child[2 * node + (right_side(xr, t, d, t[d]) ? 1 : 0)];
  }
  if (leaf) leaf[i] = node;
  if (pred) pred[i] = leaf_predict(xr, d, features[node], coef + (int64_t)node * cs);
}

// Per segment: sum of squared residuals of phi(x) . beta and sum of y^2.
// One CTA per segment; each thread walks its rows in order, then a fixed
// shared-memory tree sums the threads (deterministic for a given segment).
constexpr int kResThreads = 256;
__global__ void __launch_bounds__(kResThreads)
    residual_kernel(ArtSegments seg, const double* x, const double* y, const double* beta,
                    int64_t bs, double* sse, double* ssy) {
  const int k = blockIdx.x;
  const int64_t r0 = seg.row_offsets[k], n = seg.row_offsets[k + 1] - r0;
  const int64_t xoff = seg.x_offsets[k];
  const int d = seg.dims[k], kind = seg.features[k];
  const int p = feature_count(d, kind);
  __shared__ double b[ART_MAX_FEATURES];
  __shared__ int16_t fa[ART_MAX_FEATURES], fb[ART_MAX_FEATURES];
  __shared__ double red[2][kResThreads];
  for (int f = threadIdx.x; f < p; f += kResThreads) {
    int u, v;
    feature_factors(d, kind, f, u, v);
    fa[f] = (int16_t)u;
    fb[f] = (int16_t)v;
    b[f] = beta[(int64_t)k * bs + f];
  }
  __syncthreads();
  double s_e = 0.0, s_y = 0.0;
  for (int64_t r = threadIdx.x; r < n; r += kResThreads) {
    const double* xr = x + xoff + r * d;
    double pred = 0.0;
    for (int f = 0; f < p; ++f) {
      const int u = fa[f], v = fb[f];
      pred = fma((u < 0 ? 1.0 : xr[u]) * (v < 0 ? 1.0 : xr[v]), b[f], pred);
    }
    const double yv = y[r0 + r], e = yv - pred;
    s_e = fma(e, e, s_e);
    s_y = fma(yv, yv, s_y);
  }
  red[0][threadIdx.x] = s_e;
  red[1][threadIdx.x] = s_y;
  __syncthreads();
  for (int h = kResThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      red[0][threadIdx.x] += red[0][threadIdx.x + h];
      red[1][threadIdx.x] += red[1][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sse[k] = red[0][0];
    ssy[k] = red[1][0];
  }
}

}  // namespace
}  // namespace art

using namespace art;

extern "C" int art_segment_residuals(const ArtSegments* seg, const double* x, const double* y,
                                     const double* beta, int64_t beta_stride, double* sse,
                                     double* ssy, art_stream_t stream) {
  cudaGetLastError();
  if (!seg || seg->count < 0) { set_error("art_segment_residuals: bad segments"); return ART_E_INVALID; }
  if (seg->count == 0) return ART_OK;
  if (!seg->row_offsets || !seg->x_offsets || !seg->dims || !seg->features || !x || !y || !beta ||
      !sse || !ssy) {
    set_error("art_segment_residuals: null argument");
    return ART_E_INVALID;
  }
  if (seg->count > 0x7fffffffll) { set_error("art_segment_residuals: too many segments"); return ART_E_UNSUPPORTED; }
  prof_begin("segment_residuals", (cudaStream_t)stream);
  residual_kernel<<<(unsigned)seg->count, kResThreads, 0, (cudaStream_t)stream>>>(*seg, x, y, beta, beta_stride,
                                                                                  sse, ssy);
  prof_end((cudaStream_t)stream);
  count_launch();
  return check_launch("art_segment_residuals");
}

extern "C" int art_partition_rows(const ArtSegments* seg, const double* x, const double* theta,
                                  int64_t theta_stride, const int8_t* split, int64_t* perm,
                                  int32_t* n_right, art_stream_t stream) {
  cudaGetLastError();
  if (!seg || !x || !theta || !perm) { set_error("art_partition_rows: null argument"); return ART_E_INVALID; }
  if (seg->count < 0 || seg->count > 0x7fffffff) { set_error("art_partition_rows: bad count"); return ART_E_INVALID; }
  if (seg->count == 0) return ART_OK;
  if (theta_stride < 2) { set_error("art_partition_rows: theta_stride too small"); return ART_E_INVALID; }
  prof_begin("partition_rows", (cudaStream_t)stream);
  partition_kernel<<<(unsigned)seg->count, kPartThreads, 0, (cudaStream_t)stream>>>(
      *seg, x, theta, theta_stride, split, perm, n_right);
  prof_end((cudaStream_t)stream);
  count_launch();
  return check_launch("art_partition_rows");
}

extern "C" int art_tree_predict(int32_t dim, int64_t n_nodes, const int32_t* child,
                                const double* theta, int64_t theta_stride, const double* coef,
                                int64_t coef_stride, const int32_t* features, int64_t n_points,
                                const double* x, int32_t* leaf, double* pred, art_stream_t stream) {
  cudaGetLastError();
  if (dim < 1 || dim > ART_MAX_DIM) { set_error("art_tree_predict: bad dim %d", dim); return ART_E_UNSUPPORTED; }
  if (n_nodes < 1 || !child || !theta || !x || (pred && (!coef || !features))) {
    set_error("art_tree_predict: null argument");
    return ART_E_INVALID;
  }
  if (n_points <= 0) return ART_OK;
  const unsigned grid = (unsigned)((n_points + 255) / 256);
  prof_begin("tree_predict", (cudaStream_t)stream);
  predict_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(dim, n_nodes, child, theta, theta_stride,
                                                         coef, coef_stride, features, n_points, x,
                                                         leaf, pred);
  prof_end((cudaStream_t)stream);
  count_launch();
  return check_launch("art_tree_predict");
}
