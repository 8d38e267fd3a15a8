// abi.cu -- error reporting and launch accounting for the C ABI.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace art {

static thread_local char g_error[512];
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---- profiling: event pairs per launch, resolved lazily in report()
struct ProfRecord {
  std::string name;
  cudaEvent_t start, stop;
};
static std::atomic<int> g_prof_on{0};
static std::mutex g_prof_mu;
static std::vector<ProfRecord> g_prof_pending;
static std::vector<cudaEvent_t> g_prof_pool;
static std::map<std::string, std::pair<long, double>> g_prof_acc;
static thread_local ProfRecord t_open;
static thread_local bool t_has_open = false;

static cudaEvent_t prof_event() {
  if (!g_prof_pool.empty()) {
    cudaEvent_t e = g_prof_pool.back();
    g_prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(const char* name, cudaStream_t s) {
  if (!g_prof_on.load()) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  t_open.name = name;
  t_open.start = prof_event();
  t_open.stop = prof_event();
  cudaEventRecord(t_open.start, s);
  t_has_open = true;
}

void prof_end(cudaStream_t s) {
  if (!t_has_open) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEventRecord(t_open.stop, s);
  g_prof_pending.push_back(t_open);
  t_has_open = false;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return ART_E_LAUNCH;
  }
  return ART_OK;
}

int resident_ctas(const void* kern, int threads, size_t dyn_smem) {
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  cudaGetLastError();
  int api = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&api, kern, threads, dyn_smem) != cudaSuccess) {
    cudaGetLastError();
    api = 0;
  }
  int derived = 0;
  cudaFuncAttributes fa;
  int dev = 0;
  if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess && cudaGetDevice(&dev) == cudaSuccess) {
    int regs_sm = 65536, smem_sm = 228 * 1024, reserved = 1024, threads_sm = 2048, blocks_sm = 32;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    cudaDeviceGetAttribute(&blocks_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    const int warps = (threads + 31) / 32;
    const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;  // 256-register allocation unit
    const int by_regs = regs_warp > 0 ? (regs_sm / regs_warp) / warps : blocks_sm;
    const size_t per_block = fa.sharedSizeBytes + dyn_smem + (size_t)reserved;
    const int by_smem = per_block > 0 ? (int)((size_t)smem_sm / per_block) : blocks_sm;
    const int by_threads = threads_sm / (warps * 32);
    derived = by_regs < by_smem ? by_regs : by_smem;
    derived = derived < by_threads ? derived : by_threads;
    derived = derived < blocks_sm ? derived : blocks_sm;
  } else {
    cudaGetLastError();
  }
  const int occ = api > derived ? api : derived;
  return occ > 0 ? occ : 1;
}

}  // namespace art

extern "C" const char* art_last_error(void) { return art::g_error; }
extern "C" int art_abi_version(void) { return ART_ABI_VERSION; }
extern "C" uint64_t art_launch_count(void) { return art::g_launches.load(); }

extern "C" void art_profile_enable(int on) { art::g_prof_on.store(on ? 1 : 0); }

extern "C" void art_profile_reset(void) {
  using namespace art;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof_pending) {
    cudaEventSynchronize(r.stop);
    g_prof_pool.push_back(r.start);
    g_prof_pool.push_back(r.stop);
  }
  g_prof_pending.clear();
  g_prof_acc.clear();
}

extern "C" int art_profile_report(char* buf, size_t len) {
  using namespace art;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof_pending) {
    cudaEventSynchronize(r.stop);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.start, r.stop);
    auto& acc = g_prof_acc[r.name];
    acc.first += 1;
    acc.second += ms;
    g_prof_pool.push_back(r.start);
    g_prof_pool.push_back(r.stop);
  }
  g_prof_pending.clear();
  std::string out;
  char line[256];
  for (auto& kv : g_prof_acc) {
    snprintf(line, sizeof(line), "%s %ld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
    out += line;
  }
  if (buf && len) {
    size_t n = out.size() < len - 1 ? out.size() : len - 1;
    memcpy(buf, out.data(), n);
    buf[n] = 0;
  }
  return (int)g_prof_acc.size();
}
