// Native orchestration of rips_persistence for one point cloud.
//
// Reference: persistence.py:77-215 (rips_persistence): filtration
// (rips.py:170-200), H0 (boruvka.py, persistence.py:169-192), H1
// (reduce_h1_gpu.py), H2 (cohomology_general.py). The stages are the
// library's own entry points, called in order on one stream; intermediate
// buffers come from the stream-ordered allocator and are released together.
// The host waits only where a count decides the next allocation:
//   1. the edge count (edge buffers are sized by an estimate, rerun if short)
//   1b. on dense graphs, the exact triangle total (checked against the limit
//       before the filtration order and the forest are built)
//   2. the triangle count (and the H0 forest's status)
//   2b. with H2 on a dense complex, the tetrahedron count (checked against
//       the limit before the H1 columns are built)
//   3. the H1 reduction's status and row count (with the tetrahedron count
//      when H2 is asked for and it was not read at 2b)
//   4. the H2 reduction's status and row count
// The results stay on the device in a ph_result until copied out.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "pipeline.cuh"

using namespace ph;

struct ph_result {
  float* rows[3] = {nullptr, nullptr, nullptr};
  int64_t nrows[3] = {0, 0, 0};
  int ndim = 0;
  cudaStream_t stream = nullptr;
  int64_t stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // E, T, Q, H1 additions, H2 additions
  // the run's intermediate buffers, released (stream-ordered) by ph_result_free,
  // so that the caller's copies of the rows are queued before the frees
  std::vector<void*> scratch;
};

namespace ph {
namespace pl {

namespace detail {
constexpr int kSeqSlot = 8;  // word the readback kernel writes last
std::mutex g_slots_mu;
std::vector<Slots> g_slots_free;
std::mutex g_pinned_mu;
std::vector<Pinned> g_pinned_free;

// copies up to four device int64 values into the mapped host slots
__global__ void k_report(const int64_t* a, const int64_t* b, const int64_t* c, const int64_t* d, int count,
                         volatile int64_t* out, int64_t seq) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const int64_t* src[4] = {a, b, c, d};
  if (threadIdx.x < count && threadIdx.x < 4) out[threadIdx.x] = *src[threadIdx.x];
  __threadfence_system();
  __syncwarp();
  // the sequence word last: the host reads the values once it sees it
  if (threadIdx.x == 0) out[kSeqSlot] = seq;
  __threadfence_system();
}

// spins on the sequence word in host memory for up to half a millisecond (no
// driver call, so concurrent callers on other threads do not contend for the
// driver while waiting; the usual wait is a few microseconds, and a blocking
// wait adds its wake-up latency to every readback), then blocks
int wait_seq(const Slots& dst, int64_t seq, cudaStream_t s) {
  volatile int64_t* flag = dst.host + kSeqSlot;
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 0;; ++it) {
    if (*flag == seq) {
      std::atomic_thread_fence(std::memory_order_acquire);
      return PH_OK;
    }
    if ((it & 255) == 255 && std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(500)) break;
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    record_error(e);
    return PH_ERR_CUDA;
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return PH_OK;
}
}  // namespace detail
using namespace detail;

// Readback buffers come from a process-wide pool: a call takes one and
// returns it, so host threads that come and go (a server's worker slots) do
// not allocate pinned memory, which can wait for the whole device, on their
// first call.
Slots take_slots() {
  {
    std::lock_guard<std::mutex> lock(g_slots_mu);
    if (!g_slots_free.empty()) {
      const Slots b = g_slots_free.back();
      g_slots_free.pop_back();
      return b;
    }
  }
  void* p = nullptr;
  if (cudaHostAlloc(&p, 64 * sizeof(int64_t), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return Slots{};
  void* d = nullptr;
  if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
    cudaFreeHost(p);
    return Slots{};
  }
  Slots b{static_cast<int64_t*>(p), static_cast<int64_t*>(d), nullptr};
  b.seq = new int64_t(0);
  static_cast<int64_t*>(p)[kSeqSlot] = 0;
  return b;
}

void give_slots(const Slots& b) {
  std::lock_guard<std::mutex> lock(g_slots_mu);
  g_slots_free.push_back(b);
}

Pinned take_pinned(size_t bytes) {
  bytes = std::max<size_t>(bytes, 4096);
  {
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    // the smallest free buffer that is large enough
    int best = -1;
    for (int i = 0; i < (int)g_pinned_free.size(); ++i)
      if (g_pinned_free[i].bytes >= bytes && (best < 0 || g_pinned_free[i].bytes < g_pinned_free[best].bytes)) best = i;
    if (best >= 0) {
      const Pinned p = g_pinned_free[best];
      g_pinned_free.erase(g_pinned_free.begin() + best);
      return p;
    }
  }
  size_t sz = 4096;
  while (sz < bytes) sz <<= 1;
  Pinned p;
  if (cudaHostAlloc(&p.host, sz, cudaHostAllocPortable) != cudaSuccess) return Pinned{};
  p.bytes = sz;
  return p;
}

void give_pinned(const Pinned& p) {
  std::lock_guard<std::mutex> lock(g_pinned_mu);
  g_pinned_free.push_back(p);
}

// keeps the device's stream-ordered pool from returning memory at every sync
// (a setting of this process's pool, nothing that outlasts it). Cross-stream
// reuse stays at the default (an allocation may wait for another stream's
// free): turning it off made concurrent serving slower, through pool growth.
void keep_pool(int dev) {
  static std::once_flag once[64];
  if (dev < 0 || dev >= 64) return;
  std::call_once(once[dev], [dev]() {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  });
}

float to_f32(double v) {
  if (std::isnan(v)) return NAN;
  const double lim = 0x1p128 - 0x1p103;  // halfway between FLT_MAX and 2^128
  if (v >= lim) return INFINITY;
  if (v <= -lim) return -INFINITY;
  return (float)v;
}

int fail(int code, const std::string& msg) {
  record_message(msg.c_str());
  return code;
}

int readback(const int64_t* const* src, int count, const Slots& dst, cudaStream_t s) {
  const int64_t seq = ++*dst.seq;
  count_launch();
  if (ph::launch_pdl(k_report, dim3(1), dim3(32), 0, s, src[0], count > 1 ? src[1] : src[0],
                     count > 2 ? src[2] : src[0], count > 3 ? src[3] : src[0], count, dst.dev,
                     seq) != cudaSuccess) {
    record_error(cudaGetLastError());
    return PH_ERR_CUDA;
  }
  return wait_seq(dst, seq, s);
}

int readback_parts(const Part* parts, int nparts, const Slots& slots, cudaStream_t s) {
  for (int k = 0; k < nparts; ++k) {
    if (!parts[k].bytes) continue;
    const cudaError_t e = cudaMemcpyAsync(parts[k].dst, parts[k].src, parts[k].bytes, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) {
      record_error(e);
      return PH_ERR_CUDA;
    }
  }
  // the copies precede the report kernel in stream order: when its sequence
  // word arrives, every part is in host memory
  const int64_t seq = ++*slots.seq;
  count_launch();
  if (ph::launch_pdl(k_report, dim3(1), dim3(32), 0, s, (const int64_t*)nullptr, (const int64_t*)nullptr,
                     (const int64_t*)nullptr, (const int64_t*)nullptr, 0, slots.dev, seq) != cudaSuccess) {
    record_error(cudaGetLastError());
    return PH_ERR_CUDA;
  }
  return wait_seq(slots, seq, s);
}

i64 pool_capacity(i64 nnz, i64 K) {
  const i64 mult = nnz < (i64(1) << 24) ? 8 : 3;
  i64 cap = std::min<i64>(mult * nnz + 2 * K + (i64(1) << 23), POOL_MAX);
  // a test can make the first pool small to exercise the exhaustion retry
  const long long lim = reduce_first_pool_limit();
  if (lim > 0) cap = std::min<i64>(cap, lim);
  return cap;
}

int reduce_only(Arena& A, cudaStream_t s, const i32* off, const i32* data, i64 K, i32 col_base, i64 R,
                i32 row_base, i64 span, const uint8_t* skip, const i32* cmf, i64 pool_cap, int* status, RedOut& o) {
  o.state = A.take<i32>(K);
  o.piv = A.take<i32>(K);
  o.info = A.take<int64_t>(4);
  o.nrows = A.take<int64_t>(1);
  i32* pool = A.take<i32>(pool_cap);
  const size_t rb = ph_reduce_workspace_bytes(K, R, span);
  void* rws = A.bytes(rb);
  if (A.failed) return fail(PH_ERR_CUDA, "rips_persistence: device allocation failed");
  return ph_reduce(off, data, K, col_base, R, row_base, span, skip, cmf, o.state, o.piv, pool, pool_cap, o.info,
                   status, rws, rb, s);
}

}  // namespace pl
}  // namespace ph

using namespace ph::pl;

namespace {

// the segment record of a single cloud, and the run's counters cleared
__global__ void k_single_seg(ph_cloud_seg* seg, int64_t* blk_off, int64_t n, int32_t d, float thr_sq,
                             int64_t nblocks, int64_t* cnt) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int k = 0; k < 8; ++k) cnt[k] = 0;
  ph_cloud_seg s;
  s.pt_off = 0;
  s.vbase = 0;
  s.tile_off = 0;
  s.n = (int32_t)n;
  s.d = d;
  s.thr_sq = thr_sq;
  s.max_dim = 2;
  *seg = s;
  blk_off[0] = 0;
  blk_off[1] = nblocks;
}

// one reduction (H1 or H2) and its persistence rows, enqueued
int reduce_rows(Arena& A, cudaStream_t s, const i32* off, const i32* data, i64 K, i32 col_base, i64 R,
                i32 row_base, const uint8_t* skip, const i32* cmf, const float* filt, const i32* col_m,
                const i32* row_m, i64 pool_cap, int* status, float* rows, RedOut& o) {
  PH_TRY(reduce_only(A, s, off, data, K, col_base, R, row_base, R, skip, cmf, pool_cap, status, o));
  const size_t pb = ph_persistence_rows_workspace_bytes(K);
  void* pws = A.bytes(pb);
  if (A.failed) return fail(PH_ERR_CUDA, "rips_persistence: device allocation failed");
  return ph_persistence_rows(o.state, o.piv, K, row_base, filt, col_m, row_m, rows, o.nrows, pws, pb, s);
}

}  // namespace

extern "C" int ph_rips_persistence(const float* d_points, int64_t n, int32_t d, double max_edge_length,
                                   int32_t max_dim, int64_t max_triangles, int64_t max_tetrahedra,
                                   int32_t edge_mode, ph_result** out, void* stream) {
  if (!out) return PH_ERR_ARG;
  *out = nullptr;
  if (!d_points || n < 2 || d < 1 || max_dim < 0 || max_dim > 2 || edge_mode < 0 || edge_mode > 2 ||
      (edge_mode == 1 && d > 252))
    return fail(PH_ERR_ARG, "ph_rips_persistence: invalid argument");
  if (n >= (int64_t(1) << 31)) return fail(PH_ERR_OVERFLOW, "ph_rips_persistence: n exceeds the int32 range");
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  cudaGetDevice(&dev);
  keep_pool(dev);
  const SlotsLease lease;
  const Slots& slots = lease.b;
  if (!slots.host) return fail(PH_ERR_CUDA, "ph_rips_persistence: pinned host buffer unavailable");
  volatile int64_t* H = slots.host;

  Arena A(s);
  ph_result* res = new ph_result();
  res->stream = s;
  res->ndim = max_dim + 1;
  auto give_up = [&](int code) {
    for (float* r : res->rows)
      if (r) cudaFreeAsync(r, s);
    delete res;
    return code;
  };
  auto alloc_fail = [&]() { return give_up(fail(PH_ERR_CUDA, "ph_rips_persistence: device allocation failed")); };
  const float thr_sq = to_f32(max_edge_length * max_edge_length);

  // ---- 1. edges (rips.py:170-200; edge_kernel.py) ----------------------------------------
  const bool screened = edge_mode == 1 || (edge_mode == 0 && d >= 8 && d <= 252);
  const i64 nblocks = (n + 127) / 128;
  const i64 ntiles = ph_cloud_tiles(n);
  ph_cloud_seg* seg = A.take<ph_cloud_seg>(1);
  int64_t* blk = A.take<int64_t>(2);
  // cnt[0]: edge count; statuses as int32 words from cnt + 1: st[0] edges,
  // st[1] forest, st[2] H1 reduction, st[3] tetrahedra, st[4] H2 reduction;
  // cnt[5] triangle total, cnt[6] its work counter
  int64_t* cnt = A.take<int64_t>(8);
  if (A.failed) return alloc_fail();
  int* st = reinterpret_cast<int*>(cnt + 1);
  count_launch();
  ph::launch_pdl(k_single_seg, dim3(1), dim3(1), 0, s, seg, blk, n, d, thr_sq, nblocks, cnt);
  const size_t ews = screened ? ph_edges_screened_workspace_bytes(n, 1, d) : 0;
  void* ew = screened ? A.bytes(ews) : nullptr;
  const i64 pairs = n * (n - 1) / 2;
  // first edge buffer: 256 edges a point, 2^22 at least, and up to an eighth
  // of the pairs (at most 2^27 edges, 1.5 GiB): dense clouds (thresholds at
  // a k-NN percentile in high d keep a few percent of all pairs) then fit the
  // first pass instead of enumerating twice
  i64 cap = std::min<i64>(pairs, std::max<i64>({i64(1) << 22, 256 * n, std::min<i64>(pairs / 8, i64(1) << 27)}));
  i32 *ei = nullptr, *ej = nullptr;
  float* ed = nullptr;
  i64 E = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    cap = std::max<i64>(cap, 1);
    ei = A.take<i32>(cap);
    ej = A.take<i32>(cap);
    ed = A.take<float>(cap);
    if (A.failed) return alloc_fail();
    int rc;
    if (screened)
      rc = ph_batch_edges_enumerate_screened(d_points, seg, 1, ntiles, d, n, blk, nblocks, ei, ej, ed, cap,
                                             reinterpret_cast<unsigned long long*>(cnt), st, nullptr, ew, ews, s);
    else
      rc = ph_batch_edges_enumerate(d_points, seg, 1, ntiles, ei, ej, ed, cap,
                                    reinterpret_cast<unsigned long long*>(cnt), s);
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[2] = {cnt, cnt + 1};
    if (readback(src, 2, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_e = (int)(H[1] & 0xffffffff);
    if (st_e) return give_up(fail(st_e, "edge enumeration failed"));
    E = H[0];
    if (E <= cap || E >= (int64_t(1) << 31)) break;
    cap = E;
  }
  if (E >= (int64_t(1) << 31)) {
    char m[160];
    snprintf(m, sizeof m, "Edge count %lld exceeds int32 range; reduce max_edge_length", (long long)E);
    return give_up(fail(PH_ERR_LIMIT, m));
  }
  // the second pass ran with a buffer of the first pass's exact count; a
  // larger count now means the passes disagree, and the buffers hold only cap
  // edges, so nothing after this may read E of them
  if (E > cap) {
    char m[160];
    snprintf(m, sizeof m, "edge enumeration: %lld edges counted, buffer sized for %lld", (long long)E,
             (long long)cap);
    return give_up(fail(PH_ERR_CAPACITY, m));
  }
  res->stats[0] = E;

  // ---- 1b. dense graphs: the exact triangle total first --------------------------------------
  // On dense graphs the per-edge triangle count costs sum(deg^2), and a call
  // over the triangle limit (the reference's ValueError, with the exact total
  // in its text) needs nothing but that total: it comes from the unsorted
  // edges (an upper adjacency built by counting, no sort) and a shared-bitmap
  // pass, before the filtration order and the forest are built.
  const bool total_first = max_dim >= 1 && 4.0 * (double)E * (double)E / (double)n > 2e8 &&
                           n <= ph_triangles_total_max_vertices();
  i64 T_total = -1;
  if (total_first) {
    const size_t tt_b = ph_triangles_total_edges_workspace_bytes(E, n);
    void* tt_ws = A.bytes(tt_b);
    if (A.failed) return alloc_fail();
    const int rc = ph_triangles_total_edges(ei, ej, E, n, reinterpret_cast<unsigned long long*>(cnt + 5), tt_ws,
                                            tt_b, s);
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[1] = {cnt + 5};
    if (readback(src, 1, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    T_total = H[0];
    if (T_total > max_triangles) {
      char m[200];
      snprintf(m, sizeof m,
               "Triangle count %lld exceeds max_triangles=%lld. Reduce max_edge_length or increase max_triangles.",
               (long long)T_total, (long long)max_triangles);
      return give_up(fail(PH_ERR_LIMIT, m));
    }
  }

  // ---- 2. filtration order, adjacency, values ---------------------------------------------
  i32* si = A.take<i32>(E);
  i32* sj = A.take<i32>(E);
  float* sd = A.take<float>(E);
  i32* adj_ptr = A.take<i32>(n + 1);
  i32* adj_idx = A.take<i32>(2 * E);
  i32* adj_rank = A.take<i32>(2 * E);
  float* filt = A.take<float>(E);
  const size_t sort_b = ph_edges_sort_workspace_bytes(E), csr_b = ph_vertex_csr_workspace_bytes(E);
  void* sort_ws = A.bytes(sort_b);
  void* csr_ws = A.bytes(csr_b);
  if (A.failed) return alloc_fail();
  if (E) {
    int rc = ph_edges_sort(ei, ej, ed, E, n, si, sj, sd, sort_ws, sort_b, s);
    if (rc == PH_OK) rc = ph_vertex_csr(si, sj, E, n, adj_ptr, adj_idx, adj_rank, csr_ws, csr_b, s);
    if (rc == PH_OK) rc = ph_sqrt_f32(sd, filt, E, s);
    if (rc != PH_OK) return give_up(rc);
  } else {
    ph::zero_async(adj_ptr, sizeof(i32) * (n + 1), s);
  }

  // ---- 3. H0 (boruvka.py, persistence.py:169-192) ---------------------------------------------
  uint8_t* mask = A.take<uint8_t>(E);
  i32* comp = A.take<i32>(n);
  int64_t* ncomp = A.take<int64_t>(1);
  const size_t mst_b = ph_boruvka_workspace_bytes(n, E), h0_b = ph_h0_rows_workspace_bytes(E);
  void* mst_ws = A.bytes(mst_b);
  void* h0_ws = A.bytes(h0_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[0], sizeof(float) * 2 * n, s) != cudaSuccess)
    return alloc_fail();
  {
    int rc = ph_boruvka_mst(si, sj, E, n, mask, comp, ncomp, st + 1, mst_ws, mst_b, s);
    if (rc == PH_OK) rc = ph_h0_rows(filt, mask, E, n, res->rows[0], h0_ws, h0_b, s);
    if (rc != PH_OK) return give_up(rc);
  }
  res->nrows[0] = n;
  if (max_dim == 0) {
    const int64_t* src[1] = {cnt + 1};
    if (readback(src, 1, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_mst = (int)(H[0] >> 32);
    if (st_mst) return give_up(fail(st_mst, "ph_boruvka_mst failed"));
    A.release_to(res->scratch);
    *out = res;
    return PH_OK;
  }

  // ---- 4. triangles (triangle_kernel.py:288; reduce_h1_gpu.py:65-100) -------------------------
  int64_t* tri_off = A.take<int64_t>(E + 1);
  int64_t* tcof_off = A.take<int64_t>(E + 1);
  const size_t tc_b = ph_triangles_count_workspace_bytes(E);
  void* tc_ws = A.bytes(tc_b);
  if (A.failed) return alloc_fail();
  {
    int rc = ph_triangles_count(si, sj, E, adj_ptr, adj_idx, adj_rank, tri_off, tcof_off, tc_ws, tc_b, s);
    if (rc == PH_OK) rc = ph_max_count(tcof_off, E, cnt + 7, s);  // the longest cofacet row
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[3] = {tri_off + E, cnt + 1, cnt + 7};
    if (readback(src, 3, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
  }
  const i64 T = H[0];
  const i64 max_row = H[2];
  if ((int)(H[1] >> 32) != 0) return give_up(fail((int)(H[1] >> 32), "ph_boruvka_mst failed"));
  if (T_total >= 0 && T != T_total) {
    char m[160];
    snprintf(m, sizeof m, "triangle counts disagree: %lld per edge, %lld in total", (long long)T,
             (long long)T_total);
    return give_up(fail(PH_ERR_ARG, m));
  }
  if (T > max_triangles) {
    char m[200];
    snprintf(m, sizeof m,
             "Triangle count %lld exceeds max_triangles=%lld. Reduce max_edge_length or increase max_triangles.",
             (long long)T, (long long)max_triangles);
    return give_up(fail(PH_ERR_LIMIT, m));
  }
  if (E + 3 * T >= (int64_t(1) << 31)) {
    char m[120];
    snprintf(m, sizeof m, "Triangle count %lld exceeds the int32 rank range", (long long)T);
    return give_up(fail(PH_ERR_LIMIT, m));
  }
  res->stats[1] = T;
  i32* tri_m = A.take<i32>(T);
  i32* tri_w = A.take<i32>(T);
  i32* tri_fa = A.take<i32>(T);
  i32* tri_fb = A.take<i32>(T);
  i32* off1 = A.take<i32>(E + 1);
  i32* data1 = A.take<i32>(3 * T);
  i32* cmf1 = A.take<i32>(T);
  const size_t cc_b = ph_cofacet_csr_workspace_bytes(T, 3);
  void* cc_ws = A.bytes(cc_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[1], sizeof(float) * 2 * std::max<i64>(E, 1), s) != cudaSuccess)
    return alloc_fail();
  if (T) {
    const int rc = ph_triangles_emit(si, sj, E, adj_ptr, adj_idx, adj_rank, tri_off, tri_m, tri_w, tri_fa, tri_fb, s);
    if (rc != PH_OK) return give_up(rc);
  }
  // H2: the tetrahedron count only needs the triangles. On a dense complex
  // (T >= 16 E) it is read back here, so that a call over the tetrahedron
  // limit fails before the H1 columns are built and reduced; otherwise it is
  // launched here and read back with the H1 status (one host wait fewer)
  int64_t* tet_off = nullptr;
  i64 Q = 0;
  const bool tets_first = max_dim == 2 && T >= 16 * E;
  if (max_dim == 2) {
    tet_off = A.take<int64_t>(E + 1);
    const size_t tq_b = ph_tets_count_workspace_bytes(E);
    void* tq_ws = A.bytes(tq_b);
    if (A.failed) return alloc_fail();
    int rc = ph_tets_count(tri_off, tri_w, E, adj_ptr, adj_idx, adj_rank, nullptr, tet_off, tq_ws, tq_b, s);
    if (rc != PH_OK) return give_up(rc);
  }
  auto tets_limit = [&]() -> int {
    if (Q <= max_tetrahedra) return PH_OK;
    char m[200];
    snprintf(m, sizeof m,
             "Tetrahedra count %lld exceeds max_tetrahedra=%lld. Reduce max_edge_length or increase max_tetrahedra.",
             (long long)Q, (long long)max_tetrahedra);
    return fail(PH_ERR_LIMIT, m);
  };
  if (tets_first) {
    const int64_t* src[1] = {tet_off + E};
    if (readback(src, 1, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    Q = H[0];
    const int rc = tets_limit();
    if (rc != PH_OK) return give_up(rc);
  }
  if (T) {
    // the rows' lengths are the cofacet counts: scattered and sorted per row
    // when every row fits the shared-memory sort, else the radix form
    int rc;
    if (max_row <= ph_cofacet_rows3_max_row()) {
      const size_t r3_b = ph_cofacet_rows3_workspace_bytes(E);
      void* r3_ws = A.bytes(r3_b);
      if (A.failed) return alloc_fail();
      rc = ph_cofacet_rows3(tri_m, tri_fa, tri_fb, T, E, (i32)E, tcof_off, (int32_t)max_row, off1, data1, st + 3,
                            r3_ws, r3_b, s);
    } else {
      rc = ph_cofacet_csr(nullptr, tri_m, tri_fa, tri_fb, 3, T, E, (i32)E, off1, data1, cc_ws, cc_b, s);
    }
    if (rc == PH_OK) rc = ph_cof_max_face(nullptr, tri_m, tri_fa, tri_fb, 3, T, 0, mask, cmf1, s);
    if (rc != PH_OK) return give_up(rc);
  } else {
    ph::zero_async(off1, sizeof(i32) * (E + 1), s);
  }

  // ---- 5. H1 reduction and rows (reduce_h1_gpu.py:159-223, 574-604) --------------------------
  i64 pool1 = pool_capacity(3 * T, E);
  RedOut r1{};
  for (int attempt = 0;; ++attempt) {
    int rc = reduce_rows(A, s, off1, data1, E, 0, T, (i32)E, mask, cmf1, filt, nullptr, tri_m, pool1, st + 2,
                         res->rows[1], r1);
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[4] = {cnt + 2, r1.nrows, r1.info + 1, max_dim == 2 ? tet_off + E : r1.nrows};
    if (readback(src, 4, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_red = (int)(H[0] & 0xffffffff);
    // the word beside it: the cofacet rows' status (the tetrahedra's only later)
    if ((int)(H[0] >> 32) != 0) return give_up(fail((int)(H[0] >> 32), "ph_cofacet_rows3 failed"));
    if (st_red == PH_OK) break;
    if (st_red != PH_ERR_POOL || attempt >= 3 || pool1 >= POOL_MAX)
      return give_up(fail(st_red, "ph_reduce (H1) failed"));
    pool1 = std::min<i64>(pool1 * 4, POOL_MAX);
    ph::zero_async(st + 2, sizeof(int), s);
  }
  res->nrows[1] = H[1];
  res->stats[3] = H[2];
  if (max_dim == 2 && !tets_first) {
    Q = H[3];
    const int rc = tets_limit();
    if (rc != PH_OK) return give_up(rc);
  }
  if (max_dim == 1) {
    A.release_to(res->scratch);
    *out = res;
    return PH_OK;
  }

  // ---- 6. H2 (triangle_kernel.py:402; cohomology_general.py) --------------------------------
  if (E + T + Q >= (int64_t(1) << 31) || 4 * Q >= (int64_t(1) << 31)) {
    char m[120];
    snprintf(m, sizeof m, "Tetrahedra count %lld exceeds the int32 rank range", (long long)Q);
    return give_up(fail(PH_ERR_LIMIT, m));
  }
  res->stats[2] = Q;
  i32* tet_m = A.take<i32>(Q);
  i32* tet_faces = A.take<i32>(4 * Q);
  uint8_t* skip2 = A.take<uint8_t>(T);
  i32* cmf2 = A.take<i32>(Q);
  i32* off2 = A.take<i32>(T + 1);
  i32* data2 = A.take<i32>(4 * Q);
  // the H2 cofacet rows without a global sort when every row fits the per-row
  // sorts: a triangle's tetrahedra number at most n - 3
  const bool rows4 = n - 3 <= COF_ROWS_MAX;
  const size_t c2_b = rows4 ? cofacet_rows_aos_workspace_bytes(T) : ph_cofacet_csr_workspace_bytes(Q, 4);
  void* c2_ws = A.bytes(c2_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[2], sizeof(float) * 2 * std::max<i64>(T, 1), s) != cudaSuccess)
    return alloc_fail();
  {
    int rc = PH_OK;
    if (Q)
      rc = ph_tets_emit(si, sj, E, tri_off, tri_w, tri_fa, tri_fb, adj_ptr, adj_idx, adj_rank, nullptr, tet_off,
                        tet_m, tet_faces, st + 3, s);
    if (rc == PH_OK) rc = ph_mark_pivots(r1.state, r1.piv, E, (i32)E, skip2, T, s);
    if (rc == PH_OK && Q) rc = ph_cof_max_face(tet_faces, nullptr, nullptr, nullptr, 4, Q, (i32)E, skip2, cmf2, s);
    if (rc == PH_OK && Q)
      rc = rows4 ? cofacet_rows_aos(tet_faces, 4, Q, T, (i32)(E + T), off2, data2, st + 3, c2_ws, c2_b, s)
                 : ph_cofacet_csr(tet_faces, nullptr, nullptr, nullptr, 4, Q, T, (i32)(E + T), off2, data2, c2_ws,
                                  c2_b, s);
    if (rc != PH_OK) return give_up(rc);
    if (!Q) ph::zero_async(off2, sizeof(i32) * (T + 1), s);
  }
  i64 pool2 = pool_capacity(4 * Q, T);
  RedOut r2{};
  for (int attempt = 0;; ++attempt) {
    int rc = reduce_rows(A, s, off2, data2, T, (i32)E, Q, (i32)(E + T), skip2, cmf2, filt, tri_m, tet_m, pool2,
                         st + 4, res->rows[2], r2);
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[4] = {cnt + 2, cnt + 3, r2.nrows, r2.info + 1};
    if (readback(src, 4, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_emit = (int)(H[0] >> 32), st_red = (int)(H[1] & 0xffffffff);
    if (st_emit) return give_up(fail(st_emit, "ph_tets_emit failed"));
    if (st_red == PH_OK) break;
    if (st_red != PH_ERR_POOL || attempt >= 3 || pool2 >= POOL_MAX)
      return give_up(fail(st_red, "ph_reduce (H2) failed"));
    pool2 = std::min<i64>(pool2 * 4, POOL_MAX);
    ph::zero_async(st + 4, sizeof(int), s);
  }
  res->nrows[2] = H[2];
  res->stats[4] = H[3];
  A.release_to(res->scratch);
  *out = res;
  return PH_OK;
}

extern "C" int64_t ph_result_rows(const ph_result* r, int32_t dim) {
  if (!r || dim < 0 || dim >= r->ndim) return -1;
  return r->nrows[dim];
}

extern "C" int64_t ph_result_stat(const ph_result* r, int32_t k) {
  if (!r || k < 0 || k >= 8) return -1;
  return r->stats[k];
}

namespace {
// A copy queued on another stream than the run's: the run's stream waits for
// it, so that ph_result_free's stream-ordered frees cannot overtake it. (The
// rows themselves are complete when ph_rips_persistence returns: its last
// host wait follows them in stream order.)
int order_frees_after(const ph_result* r, cudaStream_t s) {
  if (s == r->stream) return PH_OK;
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e == cudaSuccess) {
    e = cudaEventRecord(ev, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(r->stream, ev, 0);
    cudaEventDestroy(ev);
  }
  if (e != cudaSuccess) {
    record_error(e);
    return PH_ERR_CUDA;
  }
  return PH_OK;
}
}  // namespace

extern "C" int ph_result_copy(const ph_result* r, int32_t dim, float* dst, int32_t to_host, void* stream) {
  if (!r || dim < 0 || dim >= r->ndim || (!dst && r->nrows[dim])) return PH_ERR_ARG;
  if (!r->nrows[dim]) return PH_OK;
  const cudaError_t e = cudaMemcpyAsync(dst, r->rows[dim], sizeof(float) * 2 * r->nrows[dim],
                                        to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                        (cudaStream_t)stream);
  if (e != cudaSuccess) {
    record_error(e);
    return PH_ERR_CUDA;
  }
  return order_frees_after(r, (cudaStream_t)stream);
}

extern "C" int ph_result_copy_all(const ph_result* r, float* dst, int32_t to_host, void* stream) {
  if (!r) return PH_ERR_ARG;
  int64_t at = 0;
  for (int k = 0; k < r->ndim; ++k) {
    if (r->nrows[k] && !dst) return PH_ERR_ARG;
    if (r->nrows[k]) {
      const cudaError_t e = cudaMemcpyAsync(dst + 2 * at, r->rows[k], sizeof(float) * 2 * r->nrows[k],
                                            to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                            (cudaStream_t)stream);
      if (e != cudaSuccess) {
        record_error(e);
        return PH_ERR_CUDA;
      }
    }
    at += r->nrows[k];
  }
  return at ? order_frees_after(r, (cudaStream_t)stream) : PH_OK;
}

extern "C" void ph_result_free(ph_result* r) {
  if (!r) return;
  for (float* p : r->rows)
    if (p) cudaFreeAsync(p, r->stream);
  for (void* p : r->scratch) cudaFreeAsync(p, r->stream);
  delete r;
}
