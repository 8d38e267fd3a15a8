// split_stub.cu -- placeholder until the device split-search kernel lands.
#include "common.cuh"
using namespace art;
extern "C" size_t art_split_workspace_size(int64_t, int32_t, int32_t, int32_t) { return 0; }
extern "C" int art_split_level(const ArtSplitProblem*, const ArtSplitParams*, const ArtSplitResult*,
                               void*, size_t, art_stream_t) {
  set_error("art_split_level: not built yet");
  return ART_E_UNSUPPORTED;
}
