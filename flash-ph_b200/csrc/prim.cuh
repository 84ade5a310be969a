// Device-wide primitives written for this library: exclusive scan and a
// stable LSD radix sort of (u64 key, u32 value) pairs. Both run entirely on
// the stream with no host synchronisation: the sort decides on the device
// which 8-bit digits vary and skips the passes of constant digits. Sorts of
// up to 98,304 records (16-block clusters; 49,152 with 8) run as one cluster
// launch that keeps every pass in distributed shared memory; larger ones run
// one-sweep passes through global memory.
#pragma once
#include "common.cuh"

namespace ph {

// ---- exclusive scan -------------------------------------------------------
// out[0..n] with out[n] = total. In/Out are integer types.
size_t scan_workspace_bytes(i64 n);
int scan_exclusive_i32_i32(const i32* in, i32* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s);
int scan_exclusive_i32_i64(const i32* in, i64* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s);
int scan_exclusive_u8_i32(const uint8_t* in, i32* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s);

// ---- stable radix sort -----------------------------------------------------
// Sorts keys[0..n) (and the matching vals) ascending by bits [begin_bit,
// end_bit) of the key, stably; results end in keys/vals. begin/end multiples of 8.
size_t radix_sort_workspace_bytes(i64 n);
int radix_sort_pairs(u64* keys, u32* vals, i64 n, int begin_bit, int end_bit, void* ws,
                     size_t ws_bytes, cudaStream_t s);

// Edges (i, j, dist^2), i < j < n, sorted by the packed filtration key
// bits(dist^2) << 32 | j(j-1)/2 + i into oi/oj/od in one cluster launch: the
// key is built on load and the edge rebuilt from it on store. Returns
// CLUSTER_SORT_NA (nothing launched) when E is beyond the cluster form or
// n > 92682 (the packed key is then truncated and ties need emission order).
constexpr int CLUSTER_SORT_NA = -1;
int cluster_sort_edges(const i32* ei, const i32* ej, const float* dsq, i64 E, i64 n, i32* oi, i32* oj,
                       float* od, cudaStream_t s);

// Persistence rows in the reference's order without a sort (batch.cu);
// col_off (nsegs+1 column offsets) may be null for a single segment.
size_t rows_nosort_workspace_bytes(i64 K);
int rows_nosort(const i32* state, const i32* piv, i64 K, i32 row_base, const float* filt, const i32* col_m,
                const i32* row_m, const i64* col_off, int nsegs, float* out_rows, i64* row_off, i64* d_nrows,
                void* ws, size_t ws_bytes, cudaStream_t s);

// Workspace carving helper: aligned bump allocation inside a caller buffer.
struct Carve {
  char* base;
  size_t size;
  size_t used = 0;
  Carve(void* p, size_t n) : base(static_cast<char*>(p)), size(n) {}
  template <typename T>
  T* take(i64 count) {
    size_t off = (used + 255) & ~size_t(255);
    size_t bytes = (size_t)count * sizeof(T);
    if (off + bytes > size) return nullptr;
    used = off + bytes;
    return reinterpret_cast<T*>(base + off);
  }
  static size_t need(size_t bytes) { return ((bytes + 255) & ~size_t(255)) + 256; }
};

}  // namespace ph
