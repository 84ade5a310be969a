// Host-side plumbing shared by the native whole-call pipelines (one cloud in
// pipeline.cu, a batch of clouds in batch_pipeline.cu): stream-ordered
// scratch, host readbacks of device counts and statuses, reduction-pool
// sizing and the reduction + rows step.
#pragma once
#include <algorithm>
#include <string>
#include <vector>

#include "prim.cuh"

namespace ph {
namespace pl {

// stream-ordered allocations released together when the run ends
struct Arena {
  cudaStream_t s;
  std::vector<void*> ptrs;
  bool failed = false;
  explicit Arena(cudaStream_t st) : s(st) {}
  Arena(const Arena&) = delete;
  Arena& operator=(const Arena&) = delete;
  template <typename T>
  T* take(i64 count) {
    void* p = nullptr;
    const size_t bytes = (size_t)std::max<i64>(count, 1) * sizeof(T);
    if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
      failed = true;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  void* bytes(size_t n) { return take<unsigned char>((i64)std::max<size_t>(n, 1)); }
  // hands the buffers to a result, which frees them later
  void release_to(std::vector<void*>& keep) {
    keep.swap(ptrs);
    ptrs.clear();
  }
  ~Arena() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
};

// Small pinned, device-mapped host buffers for count and status readbacks (a
// kernel writes the values into them directly), from a process-wide pool.
struct Slots {
  int64_t* host = nullptr;
  int64_t* dev = nullptr;
  int64_t* seq = nullptr;  // host-side count of readbacks through this buffer
};
Slots take_slots();
void give_slots(const Slots& b);
struct SlotsLease {
  Slots b = take_slots();
  ~SlotsLease() {
    if (b.host) give_slots(b);
  }
};

// Pinned host buffers of any size for bulk readbacks and uploads (per-cloud
// arrays of a batch), from a process-wide pool: cudaHostAlloc can wait for
// the whole device, so buffers are reused rather than allocated per call.
struct Pinned {
  void* host = nullptr;
  size_t bytes = 0;
};
Pinned take_pinned(size_t bytes);
void give_pinned(const Pinned& p);
struct PinnedLease {
  Pinned p;
  explicit PinnedLease(size_t bytes) : p(take_pinned(bytes)) {}
  PinnedLease(const PinnedLease&) = delete;
  PinnedLease& operator=(const PinnedLease&) = delete;
  ~PinnedLease() {
    if (p.host) give_pinned(p);
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p.host);
  }
};

// keeps the device's stream-ordered pool from returning memory at every sync
void keep_pool(int dev);
// fp32 of a double, round to nearest even, inf beyond the fp32 range (numpy's float32())
float to_f32(double v);
// records msg for ph_last_error() and returns code
int fail(int code, const std::string& msg);

// Brings count (<= 4) int64 values from the device into the pinned slots and
// waits (spins briefly on a sequence word written after them, then blocks).
int readback(const int64_t* const* src, int count, const Slots& dst, cudaStream_t s);
// One part of a bulk readback: bytes from device src to host dst.
struct Part {
  const void* src;
  void* dst;
  size_t bytes;
};
// Copies every part to pinned host memory (stream-ordered) and waits as
// readback does.
int readback_parts(const Part* parts, int nparts, const Slots& slots, cudaStream_t s);

// reduction pool (int32 entries): initial records (at most 2 nnz), per-warp
// chunks, reduced columns; bounded by the 33-bit record offsets
constexpr i64 POOL_MAX = (i64(1) << 33) - 1;
i64 pool_capacity(i64 nnz, i64 K);

struct RedOut {
  i32* state;
  i32* piv;
  int64_t* info;
  int64_t* nrows;
};

// One reduction (H1 or H2) enqueued on s; span as ph_reduce takes it.
int reduce_only(Arena& A, cudaStream_t s, const i32* off, const i32* data, i64 K, i32 col_base, i64 R,
                i32 row_base, i64 span, const uint8_t* skip, const i32* cmf, i64 pool_cap, int* status, RedOut& o);

}  // namespace pl
}  // namespace ph
