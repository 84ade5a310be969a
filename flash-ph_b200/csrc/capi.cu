// Library-wide C entry points: version, error reporting, launch counting.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace ph {
namespace {
thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
thread_local bool g_dependent_launch = true;
std::atomic<long long> g_reduce_max_steps{0};
std::atomic<long long> g_reduce_first_pool{0};
}  // namespace
long long reduce_max_steps() {
  const long long v = g_reduce_max_steps.load(std::memory_order_relaxed);
  return v > 0 ? v : (1ll << 24);
}
long long reduce_first_pool_limit() { return g_reduce_first_pool.load(std::memory_order_relaxed); }
void record_error(cudaError_t e) { g_last_error = cudaGetErrorString(e); }
void record_message(const char* msg) { g_last_error = msg; }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
bool dependent_launch_enabled() { return g_dependent_launch; }
// Per-device caches of launch facts that do not change while the process
// runs (attribute and occupancy queries cost a microsecond or more of host
// time each, on a path that launches dozens of kernels per call).
namespace {
std::mutex g_cache_mu;
struct FuncFact {
  int dev;
  const void* func;
  int threads;
  size_t smem;
  int value;
};
std::vector<FuncFact> g_smem_set, g_occ;
int g_sms[64] = {};
}  // namespace

int device_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!g_sms[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    g_sms[dev] = v > 0 ? v : 148;
  }
  return g_sms[dev];
}

cudaError_t allow_dynamic_smem(const void* func) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (const FuncFact& f : g_smem_set)
    if (f.dev == dev && f.func == func) return cudaSuccess;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, func);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  if (e == cudaSuccess) g_smem_set.push_back({dev, func, 0, 0, 1});
  return e;
}

namespace {
// zeroes one or two byte ranges: 16-byte stores where a range is aligned, bytes
// for its unaligned head and tail
__device__ void zero_range(uint8_t* p, size_t n) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
  const size_t head = std::min<size_t>(n, (16 - (reinterpret_cast<uintptr_t>(p) & 15)) & 15);
  for (size_t i = tid; i < head; i += nth) p[i] = 0;
  const size_t body = (n - head) / 16;
  uint4* q = reinterpret_cast<uint4*>(p + head);
  for (size_t i = tid; i < body; i += nth) q[i] = make_uint4(0, 0, 0, 0);
  for (size_t i = head + body * 16 + tid; i < n; i += nth) p[i] = 0;
}
__global__ void k_zero(uint8_t* p1, size_t n1, uint8_t* p2, size_t n2) {
  ph::pdl_wait();
  ph::pdl_trigger();
  if (p1) zero_range(p1, n1);
  if (p2) zero_range(p2, n2);
}
}  // namespace

cudaError_t zero_async(void* p1, size_t n1, cudaStream_t s, void* p2, size_t n2) {
  if (!p1) n1 = 0;
  if (!p2) n2 = 0;
  const size_t most = std::max(n1, n2);
  if (most == 0) return cudaSuccess;
  const int grid = (int)std::min<size_t>((most + 256 * 16 - 1) / (256 * 16), 296);
  count_launch();
  return launch_pdl(k_zero, dim3(grid), dim3(256), 0, s, static_cast<uint8_t*>(p1), n1, static_cast<uint8_t*>(p2), n2);
}

int occupancy(const void* func, int threads, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(g_cache_mu);
  for (const FuncFact& f : g_occ)
    if (f.dev == dev && f.func == func && f.threads == threads && f.smem == smem) return f.value;
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, func, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  g_occ.push_back({dev, func, threads, smem, v});
  return v;
}
}  // namespace ph

extern "C" int ph_version(void) { return 100; }

extern "C" const char* ph_last_error(void) { return ph::g_last_error.c_str(); }

extern "C" unsigned long long ph_launch_count(void) {
  return ph::g_launches.load(std::memory_order_relaxed);
}

extern "C" void ph_set_dependent_launch(int32_t enable) { ph::g_dependent_launch = enable != 0; }

extern "C" void ph_set_reduce_limits(int64_t max_steps, int64_t first_pool_entries) {
  ph::g_reduce_max_steps.store(max_steps > 0 ? max_steps : 0, std::memory_order_relaxed);
  ph::g_reduce_first_pool.store(first_pool_entries > 0 ? first_pool_entries : 0, std::memory_order_relaxed);
}

// ---- a measurement probe: the latency of one dependent L2 load ------------------------
namespace {
// One thread follows a chain of indices through `next` (a random cycle over a
// buffer that fits L2): every load's address depends on the previous load, as
// the reducer's owner-word and record loads do. A first lap over the same
// addresses warms L2; the second is timed.
__global__ void k_chase(const uint32_t* __restrict__ next, int hops, uint32_t start, unsigned long long* out) {
  uint32_t w = start;
  for (int i = 0; i < hops; ++i) w = __ldcg(next + w);
  uint32_t p = start;
  unsigned long long t0, t1;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0)::"memory");
  for (int i = 0; i < hops; ++i) p = __ldcg(next + p);
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1)::"memory");
  out[0] = t1 - t0;
  out[1] = (unsigned long long)p + w;  // keeps both chains live
}
}  // namespace

extern "C" int ph_probe_l2_chase(const uint32_t* next, int32_t hops, uint32_t start, unsigned long long* d_out,
                                 void* stream) {
  if (!next || !d_out || hops < 1) return PH_ERR_ARG;
  ph::count_launch();
  k_chase<<<1, 1, 0, (cudaStream_t)stream>>>(next, hops, start, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ph::record_error(e);
    return PH_ERR_CUDA;
  }
  return PH_OK;
}
