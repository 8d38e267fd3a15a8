// ridge_tc.cu -- mixed-precision (tcgen05) ridge path.  Placeholder until the
// tensor-core kernel lands: the mixed form is rejected explicitly.
#include "ridge.cuh"
namespace art {
int launch_ridge_tensor(const RidgeArgs&, const RidgeLists&, cudaStream_t) {
  set_error("art_ridge_batched: the mixed-precision form is not built yet");
  return ART_E_UNSUPPORTED;
}
}  // namespace art
