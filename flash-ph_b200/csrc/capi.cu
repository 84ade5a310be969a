// Library-wide C entry points: version, error reporting, launch counting.
#include <atomic>
#include <string>

#include "common.cuh"

namespace ph {
namespace {
thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
}  // namespace
void record_error(cudaError_t e) { g_last_error = cudaGetErrorString(e); }
void record_message(const char* msg) { g_last_error = msg; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
cudaError_t allow_dynamic_smem(const void* func) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, func);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  return e;
}
}  // namespace ph

extern "C" int ph_version(void) { return 100; }

extern "C" const char* ph_last_error(void) { return ph::g_last_error.c_str(); }

extern "C" unsigned long long ph_launch_count(void) {
  return ph::g_launches.load(std::memory_order_relaxed);
}
