// Filtration sort for callers that cannot allocate device memory.
//
// Some callers own all of their device memory through another allocator --
// a framework's caching allocator, or a serving process that reserves a
// fixed HBM budget up front -- and must not call cudaMalloc behind its back.
// ph_edges_sort_noalloc() gives them the filtration sort of ph_edges_sort()
// with no allocation at all: the caller passes only inputs and outputs, and
// the scratch lives in the file-scope device array below (13 MiB, enough for
// up to 2^19 edges). Every GPU that loads this library holds the array until
// the process exits.
//
// The host cannot use the array's name as a device address, so the address
// is looked up with cudaGetSymbolAddress once per device, on the first call
// made while that device is current, and cached. All calls on a device share
// the one array and it keeps the last call's contents; the sort clears the
// parts that must start at zero (its control block and look-back flags) on
// every call. Two calls whose work overlaps on the GPU (for instance on two
// streams at once) race on the array; callers must order them.
#include <mutex>

#include "prim.cuh"

namespace {

constexpr int64_t kNoAllocMaxEdges = int64_t(1) << 19;
constexpr size_t kNoAllocScratchBytes = size_t(13) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_sort_scratch on the current device (set-up on first use).
int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    ph::record_error(e);
    return PH_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return PH_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
      ph::record_error(e);
      return PH_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return PH_OK;
}

}  // namespace

extern "C" int64_t ph_edges_sort_noalloc_max_edges(void) { return kNoAllocMaxEdges; }

extern "C" int ph_edges_sort_noalloc(const int32_t* in_i, const int32_t* in_j, const float* in_dsq,
                                     int64_t E, int64_t n, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                     void* stream) {
  if (E < 0 || n < 0) return PH_ERR_ARG;
  if (E > kNoAllocMaxEdges || ph_edges_sort_workspace_bytes(E) > kNoAllocScratchBytes) {
    ph::record_message("ph_edges_sort_noalloc: edge count exceeds the fixed scratch maximum of 524288 edges");
    return PH_ERR_CAPACITY;
  }
  void* scratch = nullptr;
  PH_TRY(scratch_for_current_device(&scratch));
  return ph_edges_sort(in_i, in_j, in_dsq, E, n, out_i, out_j, out_dsq, scratch, kNoAllocScratchBytes,
                       stream);
}
