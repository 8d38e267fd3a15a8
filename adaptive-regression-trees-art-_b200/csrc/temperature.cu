// temperature.cu -- batched median nearest-neighbour distance, the "median_nn"
// temperature scale of the split search (temperature.py:73-137).
//
// One CTA per point set (at most ART_MEDIAN_NN_MAX_SET points, drawn by the
// host).  Each thread takes points i = tid, tid + 256, ... and scans every
// other point of the set for the nearest one: squared distances summed over
// the coordinates in order with separate roundings, the minimum taken, then
// one square root (the square root is monotone, so this is the minimum
// distance).  The set's distances are ranked in shared memory (ties broken
// by index) to place each at its sorted position, and the median is the
// middle value, or the mean of the two middle values for an even count, as
// numpy's median.  The result is c * median.  A set larger than the
// caller's max_set (which sized the shared arrays) gives NaN, as a set of
// fewer than two points does, and touches no shared memory.
#include "common.cuh"

namespace art {
namespace {

constexpr int kTempThreads = 256;

__global__ void __launch_bounds__(kTempThreads) median_nn_kernel(int64_t count, const double* x,
                                                                 const int64_t* x_offsets,
                                                                 const int32_t* dims,
                                                                 const int64_t* sample_offsets,
                                                                 const int64_t* sample_rows, int max_set,
                                                                 double c, double* out) {
  extern __shared__ double s_nn[];  // [max_set] distances, then [max_set] sorted
  const int tid = threadIdx.x;
  for (int64_t k = blockIdx.x; k < count; k += gridDim.x) {
    const int64_t s0 = sample_offsets[k];
    const int m = (int)(sample_offsets[k + 1] - s0);
    const int d = dims[k];
    // fewer than two points, or more than the shared arrays were sized for
    // (a caller's max_set below its largest set): NaN, and no shared access
    if (m < 2 || m > max_set) {
      if (tid == 0) out[k] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    const double* X = x + x_offsets[k];
    const int64_t* rows = sample_rows + s0;
    double* nn = s_nn;
    double* sorted = s_nn + m;
    for (int i = tid; i < m; i += kTempThreads) {
      const double* xi = X + rows[i] * d;
      double best = __longlong_as_double(0x7ff0000000000000ll);  // +inf
      for (int j = 0; j < m; ++j) {
        if (j == i) continue;
        const double* xj = X + rows[j] * d;
        double s = 0.0;
        for (int t = 0; t < d; ++t) {
          const double diff = __dsub_rn(xi[t], xj[t]);
          s = __dadd_rn(s, __dmul_rn(diff, diff));
        }
        best = fmin(best, s);
      }
      nn[i] = sqrt(best);
    }
    __syncthreads();
    for (int i = tid; i < m; i += kTempThreads) {
      const double v = nn[i];
      int rank = 0;
      for (int j = 0; j < m; ++j) {
        const double u = nn[j];
        rank += (u < v || (u == v && j < i)) ? 1 : 0;
      }
      sorted[rank] = v;
    }
    __syncthreads();
    if (tid == 0) {
      const double med = (m & 1) ? sorted[m / 2] : (sorted[m / 2 - 1] + sorted[m / 2]) / 2.0;
      out[k] = c * med;
    }
    __syncthreads();  // the next set reuses the shared arrays
  }
}

}  // namespace
}  // namespace art

using namespace art;

extern "C" int art_median_nn_distance(
    int64_t count, const double* x, const int64_t* x_offsets, const int32_t* dims,
    const int64_t* sample_offsets, const int64_t* sample_rows, int32_t max_set, double c,
    double* temperature, art_stream_t stream) {
  if (count < 0) { set_error("art_median_nn_distance: negative count"); return ART_E_INVALID; }
  if (count == 0) return ART_OK;
  if (!x || !x_offsets || !dims || !sample_offsets || !sample_rows || !temperature) {
    set_error("art_median_nn_distance: null device pointer");
    return ART_E_INVALID;
  }
  if (!(c > 0.0)) { set_error("art_median_nn_distance: c must be positive"); return ART_E_INVALID; }
  if (max_set < 0 || max_set > ART_MEDIAN_NN_MAX_SET) {
    set_error("art_median_nn_distance: max_set must be in [0, %d]", ART_MEDIAN_NN_MAX_SET);
    return ART_E_UNSUPPORTED;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t smem = (size_t)2 * (max_set > 2 ? max_set : 2) * sizeof(double);
  if (cudaFuncSetAttribute(median_nn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    set_error("art_median_nn_distance: cannot reserve %zu bytes of shared memory", smem);
    return ART_E_UNSUPPORTED;
  }
  const int64_t grid = count < 65535 ? count : 65535;
  prof_begin("median_nn", s);
  median_nn_kernel<<<(unsigned)grid, kTempThreads, smem, s>>>(count, x, x_offsets, dims, sample_offsets,
                                                              sample_rows, max_set, c, temperature);
  prof_end(s);
  count_launch();
  return check_launch("median_nn");
}
