// Shared definitions for the flash-ph B200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/flashph_b200.h"

namespace ph {

using i32 = int32_t;
using i64 = int64_t;
using u32 = uint32_t;
using u64 = uint64_t;

constexpr int kWarp = 32;

inline int ceil_div(i64 a, i64 b) { return (int)((a + b - 1) / b); }

// Records the first device-side error code; later codes do not overwrite it.
__device__ __forceinline__ void set_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ u32 float_bits(float f) { return __float_as_uint(f); }

// Remembers the message of a failed CUDA call for ph_last_error().
void record_error(cudaError_t e);
// Remembers a library-side error message for ph_last_error().
void record_message(const char* msg);

// Counts kernel launches made by this library (reported by ph_launch_count()).
void count_launch();
// The reducer's step cap per column (ph_set_reduce_limits; 2^24 by default)
// and the cap on a native call's first reduction pool (0: none).
long long reduce_max_steps();
// the cofacet CSR of simplices given as k faces each, without a global sort (simplices.cu)
constexpr int COF_ROWS_MAX = 8192;  // longest row the per-row sorts take
size_t cofacet_rows_aos_workspace_bytes(int64_t n_faces);
int cofacet_rows_aos(const int32_t* faos, int32_t k, int64_t S, int64_t n_faces, int32_t row_base, int32_t* cof_off,
                     int32_t* cof_data, int* d_status, void* workspace, size_t workspace_bytes, cudaStream_t s);
// the triangle count pass with an optional per-cloud mask (simplices.cu)
int triangles_count_masked(const int32_t* edge_i, const int32_t* edge_j, int64_t E, const int32_t* adj_ptr,
                           const int32_t* adj_idx, const int32_t* adj_rank, int64_t* tri_off, int64_t* cof_off,
                           void* workspace, size_t workspace_bytes, const uint8_t* keep, const int32_t* vcloud,
                           cudaStream_t s);
long long reduce_first_pool_limit();

// Raises a kernel's dynamic shared memory limit to the device's opt-in
// maximum (minus the kernel's static shared memory). Always the same value,
// so threads launching the kernel concurrently with different requests
// cannot lower each other's limit. Returns cudaSuccess or the error.
cudaError_t allow_dynamic_smem(const void* func);
// Zeroes n1 bytes at p1 (and n2 bytes at p2) with one kernel launched like
// every other (a memset node would end the chain of dependent launches).
cudaError_t zero_async(void* p1, size_t n1, cudaStream_t s, void* p2 = nullptr, size_t n2 = 0);
// SM count of the current device (cached)
int device_sms();
// resident blocks per SM of func at this block size and dynamic shared
// memory (cached; 0 when the query fails)
int occupancy(const void* func, int threads, size_t smem);

// Programmatic dependent launch. Kernels are launched with launch_pdl(), so
// that the next kernel in the stream is scheduled while the current one
// drains instead of after it (the launch latency between the ~80 short
// kernels of a call is hidden). Every kernel starts with pdl_wait(), which
// returns once the previous grid in the stream has completed and its memory
// is visible (a no-op for a kernel not launched that way), and then lets its
// own successor be scheduled with pdl_trigger(): the successor still waits in
// its own pdl_wait() for this grid to complete.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Whether launches from the calling host thread use dependent launch (on by
// default; ph_set_dependent_launch switches it per thread).
bool dependent_launch_enabled();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = dependent_launch_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace ph

#define PH_CHECK_LAUNCH()                         \
  do {                                            \
    cudaError_t _e = cudaGetLastError();          \
    if (_e != cudaSuccess) {                      \
      ph::record_error(_e);                       \
      return PH_ERR_CUDA;                         \
    }                                             \
  } while (0)

#define PH_TRY(expr)                  \
  do {                                \
    int _rc = (expr);                 \
    if (_rc != PH_OK) return _rc;     \
  } while (0)
