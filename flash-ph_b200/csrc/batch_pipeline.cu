// Native orchestration of rips_persistence for a batch of point clouds.
//
// The reference has no batched API: it is rips_persistence (persistence.py
// :77-215) called once per cloud. Here a batch is the disjoint union of its
// clouds (cloud c's vertex v is global vertex vbase_c + v) and the whole call
// is one library entry point: the clouds' points are gathered into one
// buffer, every stage runs once over the union on one stream (edges per
// (cloud, tile) work item, the filtration sort per cloud then by cloud, the
// adjacency, forest, triangles, tetrahedra and reductions on global indices,
// since no simplex spans two clouds), and the rows are cut per cloud. The
// host waits four times whatever the number of clouds:
//   1. the edge count,
//   2. the per-cloud triangle counts (the reference's max_triangles check per
//      cloud, and the rank range of the union),
//   3. the H1 status and row offsets, with the per-cloud tetrahedron counts
//      when some cloud asks for H2,
//   4. the H2 status and row offsets.
// A cloud over a limit gets the reference's ValueError text as its status and
// its later stages are masked out (its triangles or tetrahedra are not
// emitted, its columns are skipped); the others are unaffected. Every cloud's
// diagrams equal those of ph_rips_persistence on it alone, bit for bit.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "pipeline.cuh"

using namespace ph;
using namespace ph::pl;

struct ph_batch_result {
  int nclouds = 0;
  cudaStream_t stream = nullptr;
  std::vector<int32_t> status;        // per cloud: PH_OK or PH_ERR_LIMIT
  std::vector<std::string> message;   // per cloud: the ValueError text of a limit
  std::vector<int64_t> stat[3];       // per cloud: edges, triangles, tetrahedra (-1: not counted)
  float* rows[3] = {nullptr, nullptr, nullptr};
  std::vector<int64_t> off[3];        // per dim: nclouds + 1 row offsets into rows[dim]
  std::vector<void*> scratch;
};

namespace {

struct GatherItem {
  const float* src;
  int64_t dst_off;  // floats
  int64_t count;    // floats
};

// every cloud's points into the union buffer: a grid-stride walk over all
// floats of the batch, each element's cloud found by binary search in the
// clouds' destination offsets (items are in destination order), four
// independent copies per thread in flight
__global__ void k_gather_points(const GatherItem* __restrict__ items, int nclouds, i64 total,
                                float* __restrict__ dst) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 x0 = (i64)blockIdx.x * blockDim.x + threadIdx.x; x0 < total; x0 += 4 * stride) {
    float v[4];
    i64 at[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const i64 x = x0 + q * stride;
      at[q] = x;
      if (x >= total) continue;
      int lo = 0, hi = nclouds - 1;  // last cloud with dst_off <= x
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].dst_off <= x) lo = mid;
        else hi = mid - 1;
      }
      v[q] = items[lo].src[x - items[lo].dst_off];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (at[q] < total) dst[at[q]] = v[q];
  }
}

__global__ void k_zero_i64(int64_t* p, int n) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0;
}

// out[c] = off[item_off[c + 1]] - off[item_off[c]]: the per-cloud totals of
// per-item counts given by their exclusive scan
__global__ void k_seg_diff(const int64_t* __restrict__ off, const int64_t* __restrict__ item_off, int nsegs,
                           int64_t* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nsegs; c += gridDim.x * blockDim.x)
    out[c] = off[item_off[c + 1]] - off[item_off[c]];
}

// out[c] = off[item_off[c]] for c = 0..nsegs
__global__ void k_gather_off(const int64_t* __restrict__ off, const int64_t* __restrict__ item_off, int nsegs,
                             int64_t* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= nsegs; c += gridDim.x * blockDim.x)
    out[c] = off[item_off[c]];
}

// out[e] = (base ? base[e] : 0) | (flag of edge e's cloud, negated when invert)
__global__ void k_edge_flags(const i32* __restrict__ si, i64 E, const i32* __restrict__ vcloud,
                             const uint8_t* __restrict__ cloud_flag, int invert, const uint8_t* __restrict__ base,
                             uint8_t* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const uint8_t f = cloud_flag[vcloud[si[e]]];
    out[e] = (uint8_t)((base ? base[e] : 0) | (invert ? !f : (f != 0)));
  }
}

// cnt[e] = keep[e] ? off[e + 1] - off[e] : 0 (to be scanned again)
__global__ void k_masked_counts(const int64_t* __restrict__ off, i64 E, const uint8_t* __restrict__ keep,
                                i32* __restrict__ cnt) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x)
    cnt[e] = keep[e] ? (i32)(off[e + 1] - off[e]) : 0;
}

// Clouds that may hold more than max_triangles triangles: a graph with m
// edges has at most sqrt(2)/3 m^1.5 of them, so only clouds with more than
// m_star edges are counted exactly before the per-edge pass.
__global__ void k_tri_want(const int64_t* __restrict__ e_off, int K, i64 m_star, uint8_t* __restrict__ want) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < K; c += gridDim.x * blockDim.x)
    want[c] = (uint8_t)(e_off[c + 1] - e_off[c] > m_star);
}

// the clouds whose triangles the per-edge pass counts: all but those counted
// exactly and over the limit
__global__ void k_tri_keep(const uint8_t* __restrict__ want, const unsigned long long* __restrict__ tot, int K,
                           i64 max_t, uint8_t* __restrict__ keep) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < K; c += gridDim.x * blockDim.x)
    keep[c] = (uint8_t)!(want[c] && tot[c] > (unsigned long long)max_t);
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}

// the per-item offsets `off` (E + 1) with the items of cleared clouds removed
int mask_offsets(Arena& A, cudaStream_t s, int64_t* off, i64 E, const uint8_t* keep_edge) {
  i32* cnt = A.take<i32>(E + 1);
  const size_t sb = scan_workspace_bytes(E);
  void* sws = A.bytes(sb);
  if (A.failed) return fail(PH_ERR_CUDA, "rips_persistence_batch: device allocation failed");
  if (E > 0) {
    count_launch();
    ph::launch_pdl(k_masked_counts, dim3(grid_for(E)), dim3(256), 0, s, (const int64_t*)off, E, keep_edge, cnt);
  }
  return scan_exclusive_i32_i64(cnt, off, E, sws, sb, s);
}

std::string tri_limit_msg(i64 T, i64 cap) {
  char m[200];
  snprintf(m, sizeof m,
           "Triangle count %lld exceeds max_triangles=%lld. Reduce max_edge_length or increase max_triangles.",
           (long long)T, (long long)cap);
  return m;
}

std::string tet_limit_msg(i64 Q, i64 cap) {
  char m[200];
  snprintf(m, sizeof m,
           "Tetrahedra count %lld exceeds max_tetrahedra=%lld. Reduce max_edge_length or increase max_tetrahedra.",
           (long long)Q, (long long)cap);
  return m;
}

}  // namespace

extern "C" int ph_rips_persistence_batch(const float* const* points, const int64_t* n, const int32_t* d,
                                         const double* max_edge_length, const int32_t* max_dim, int32_t nclouds,
                                         int64_t max_triangles, int64_t max_tetrahedra, int32_t edge_mode,
                                         int64_t max_batch_simplices, ph_batch_result** out, void* stream) {
  if (!out) return PH_ERR_ARG;
  *out = nullptr;
  if (nclouds < 1 || !points || !n || !d || !max_edge_length || !max_dim || edge_mode < 0 || edge_mode > 2)
    return fail(PH_ERR_ARG, "ph_rips_persistence_batch: invalid argument");
  const int K = nclouds;
  i64 N = 0, floats = 0, pairs = 0, ntiles = 0, nblocks = 0;
  int max_d = 1, dim_all = 0;
  bool any_wrap = false;
  std::vector<ph_cloud_seg> segs(K);
  std::vector<GatherItem> gather(K);
  std::vector<int64_t> blk(K + 1, 0);
  for (int c = 0; c < K; ++c) {
    if (!points[c] || n[c] < 2 || d[c] < 1 || max_dim[c] < 0 || max_dim[c] > 2 || !(max_edge_length[c] >= 0) ||
        (max_dim[c] == 2 && n[c] >= 65536))
      return fail(PH_ERR_ARG, "ph_rips_persistence_batch: invalid cloud " + std::to_string(c));
    segs[c].pt_off = floats;
    segs[c].vbase = N;
    segs[c].tile_off = ntiles;
    segs[c].n = (int32_t)n[c];
    segs[c].d = d[c];
    segs[c].thr_sq = to_f32(max_edge_length[c] * max_edge_length[c]);
    segs[c].max_dim = max_dim[c];
    gather[c] = GatherItem{points[c], floats, n[c] * d[c]};
    floats += n[c] * d[c];
    N += n[c];
    pairs += n[c] * (n[c] - 1) / 2;
    ntiles += ph_cloud_tiles(n[c]);
    blk[c + 1] = blk[c] + (n[c] + 127) / 128;
    max_d = std::max(max_d, (int)d[c]);
    dim_all = std::max(dim_all, (int)max_dim[c]);
    any_wrap = any_wrap || n[c] > 92682;
  }
  nblocks = blk[K];
  if (N >= (int64_t(1) << 31)) return fail(PH_ERR_OVERFLOW, "ph_rips_persistence_batch: too many points");
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  cudaGetDevice(&dev);
  keep_pool(dev);
  const SlotsLease lease;
  const Slots& slots = lease.b;
  if (!slots.host) return fail(PH_ERR_CUDA, "ph_rips_persistence_batch: pinned host buffer unavailable");
  volatile int64_t* H = slots.host;

  Arena A(s);
  ph_batch_result* res = new ph_batch_result();
  res->nclouds = K;
  res->stream = s;
  res->status.assign(K, PH_OK);
  res->message.assign(K, std::string());
  for (auto& v : res->stat) v.assign(K, -1);
  auto give_up = [&](int code) {
    for (float* r : res->rows)
      if (r) cudaFreeAsync(r, s);
    delete res;
    return code;
  };
  auto alloc_fail = [&]() { return give_up(fail(PH_ERR_CUDA, "ph_rips_persistence_batch: device allocation failed")); };

  // ---- upload: segment table, gather table, block offsets (one copy) ----------------------
  const size_t seg_b = sizeof(ph_cloud_seg) * K, gat_b = sizeof(GatherItem) * K, blk_b = sizeof(int64_t) * (K + 1);
  const size_t up_b = ((seg_b + 15) & ~size_t(15)) + ((gat_b + 15) & ~size_t(15)) + blk_b;
  PinnedLease up(up_b + 16 * (size_t)K + 64);
  if (!up.p.host) return give_up(fail(PH_ERR_CUDA, "ph_rips_persistence_batch: pinned host buffer unavailable"));
  char* uh = up.as<char>();
  const size_t gat_at = (seg_b + 15) & ~size_t(15), blk_at = gat_at + ((gat_b + 15) & ~size_t(15));
  memcpy(uh, segs.data(), seg_b);
  memcpy(uh + gat_at, gather.data(), gat_b);
  memcpy(uh + blk_at, blk.data(), blk_b);
  char* ud = static_cast<char*>(A.bytes(up_b));
  float* pts = A.take<float>(floats);
  i32* vcloud = A.take<i32>(N);
  int64_t* cnt = A.take<int64_t>(16);
  if (A.failed) return alloc_fail();
  const ph_cloud_seg* dsegs = reinterpret_cast<const ph_cloud_seg*>(ud);
  const GatherItem* dgat = reinterpret_cast<const GatherItem*>(ud + gat_at);
  const int64_t* dblk = reinterpret_cast<const int64_t*>(ud + blk_at);
  if (cudaMemcpyAsync(ud, uh, up_b, cudaMemcpyHostToDevice, s) != cudaSuccess) {
    record_error(cudaGetLastError());
    return give_up(PH_ERR_CUDA);
  }
  // st[0] edges, [1] forest, [2] H1, [3] tetrahedra, [4] H2, [5] cofacet rows
  int* st = reinterpret_cast<int*>(cnt + 1);
  count_launch();
  ph::launch_pdl(k_zero_i64, dim3(1), dim3(32), 0, s, cnt, 16);
  count_launch();
  ph::launch_pdl(k_gather_points, dim3((unsigned)std::max<i64>(1, std::min<i64>((floats + 1023) / 1024, 148 * 16))),
                 dim3(256), 0, s, dgat, K, floats, pts);
  PH_TRY(ph_batch_vertex_cloud(dsegs, K, vcloud, s));

  // ---- 1. edges --------------------------------------------------------------------------------
  const bool screened = max_d <= 252 && (edge_mode == 1 || (edge_mode == 0 && max_d >= 8));
  const size_t ews = screened ? ph_edges_screened_workspace_bytes(N, K, max_d) : 0;
  void* ew = screened ? A.bytes(ews) : nullptr;
  i64 cap = std::min<i64>(pairs, std::max<i64>({i64(1) << 22, 256 * N, std::min<i64>(pairs / 8, i64(1) << 27)}));
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
      rc = ph_batch_edges_enumerate_screened(pts, dsegs, K, ntiles, max_d, N, dblk, nblocks, ei, ej, ed, cap,
                                             reinterpret_cast<unsigned long long*>(cnt), st, nullptr, ew, ews, s);
    else
      rc = ph_batch_edges_enumerate(pts, dsegs, K, ntiles, ei, ej, ed, cap, reinterpret_cast<unsigned long long*>(cnt),
                                    s);
    if (rc != PH_OK) return give_up(rc);
    const int64_t* src[2] = {cnt, cnt + 1};
    if (readback(src, 2, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_e = (int)(H[1] & 0xffffffff);
    if (st_e) return give_up(fail(st_e, "edge enumeration failed"));
    E = H[0];
    if (E <= cap || E >= (int64_t(1) << 31)) break;
    cap = E;
  }
  if (E >= (int64_t(1) << 31)) return give_up(fail(PH_ERR_CAPACITY, "ph_rips_persistence_batch: union edge count exceeds the int32 range"));
  if (E > cap) return give_up(fail(PH_ERR_CAPACITY, "ph_rips_persistence_batch: edge counts of the two passes differ"));

  // ---- 2. filtration order per cloud, adjacency, values ------------------------------------------
  i32* si = A.take<i32>(E);
  i32* sj = A.take<i32>(E);
  float* sd = A.take<float>(E);
  int64_t* e_off = A.take<int64_t>(K + 1);
  i32* adj_ptr = A.take<i32>(N + 1);
  i32* adj_idx = A.take<i32>(2 * E);
  i32* adj_rank = A.take<i32>(2 * E);
  float* filt = A.take<float>(E);
  const size_t sort_b = ph_batch_edges_sort_workspace_bytes(E), csr_b = ph_vertex_csr_workspace_bytes(E);
  void* sort_ws = A.bytes(sort_b);
  void* csr_ws = A.bytes(csr_b);
  if (A.failed) return alloc_fail();
  if (E) {
    int rc = ph_batch_edges_sort(ei, ej, ed, E, vcloud, dsegs, K, any_wrap ? 1 : 0, si, sj, sd, sort_ws, sort_b, s);
    if (rc == PH_OK) rc = ph_vertex_csr(si, sj, E, N, adj_ptr, adj_idx, adj_rank, csr_ws, csr_b, s);
    if (rc == PH_OK) rc = ph_sqrt_f32(sd, filt, E, s);
    if (rc != PH_OK) return give_up(rc);
  } else {
    ph::zero_async(adj_ptr, sizeof(i32) * (N + 1), s);
  }
  PH_TRY(ph_batch_item_offsets(si, E, vcloud, K, e_off, s));

  // ---- 3. H0 per cloud ----------------------------------------------------------------------------
  uint8_t* mask = A.take<uint8_t>(E);
  i32* comp = A.take<i32>(N);
  int64_t* ncomp = A.take<int64_t>(1);
  const size_t mst_b = ph_boruvka_workspace_bytes(N, E), h0_b = ph_batch_h0_rows_workspace_bytes(E);
  void* mst_ws = A.bytes(mst_b);
  void* h0_ws = A.bytes(h0_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[0], sizeof(float) * 2 * N, s) != cudaSuccess) return alloc_fail();
  {
    int rc = ph_boruvka_mst(si, sj, E, N, mask, comp, ncomp, st + 1, mst_ws, mst_b, s);
    if (rc == PH_OK) rc = ph_batch_h0_rows(filt, mask, E, e_off, dsegs, K, vcloud, N, res->rows[0], h0_ws, h0_b, s);
    if (rc != PH_OK) return give_up(rc);
  }
  res->off[0].resize(K + 1);
  for (int c = 0; c <= K; ++c) res->off[0][c] = c < K ? segs[c].vbase : N;

  // per-cloud host arrays read back in bulk: [0, K] edge offsets, then K counts
  PinnedLease hb(sizeof(int64_t) * (6 * (size_t)K + 8) + 256);
  if (!hb.p.host) return give_up(fail(PH_ERR_CUDA, "ph_rips_persistence_batch: pinned host buffer unavailable"));
  int64_t* hcnt = hb.as<int64_t>();            // 16 words of cnt
  int64_t* hoff = hcnt + 16;                  // K + 1 offsets
  int64_t* hper = hoff + (K + 1);             // K per-cloud counts
  int64_t* hoff2 = hper + K;                  // K + 1 more offsets
  int64_t* htot = hoff2 + (K + 1);            // K exact totals of the clouds that may be over the limit
  uint8_t* hwant = reinterpret_cast<uint8_t*>(htot + K);  // K flags: which clouds those are

  if (dim_all == 0) {
    Part parts[2] = {{cnt, hcnt, 16 * sizeof(int64_t)}, {e_off, hoff, sizeof(int64_t) * (K + 1)}};
    if (readback_parts(parts, 2, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_mst = (int)(hcnt[1] >> 32);
    if (st_mst) return give_up(fail(st_mst, "ph_boruvka_mst failed"));
    for (int c = 0; c < K; ++c) res->stat[0][c] = hoff[c + 1] - hoff[c];
    A.release_to(res->scratch);
    *out = res;
    return PH_OK;
  }

  // ---- 4. triangles: per-cloud counts, the limit per cloud ----------------------------------------
  int64_t* tri_off = A.take<int64_t>(E + 1);
  int64_t* tcof_off = A.take<int64_t>(E + 1);
  int64_t* per = A.take<int64_t>(K);
  uint8_t* cflag = A.take<uint8_t>(2 * K);  // per-cloud flags: [0, K) H1 kept, [K, 2K) H2 kept
  uint8_t* eflag = A.take<uint8_t>(E);
  const size_t tc_b = ph_triangles_count_workspace_bytes(E);
  void* tc_ws = A.bytes(tc_b);
  // clouds that may be over max_triangles are counted exactly first (the
  // bitmap total: far cheaper than the per-edge pass on a dense cloud), and
  // the per-edge pass skips those over it
  uint8_t* want = A.take<uint8_t>(K);
  uint8_t* tkeep = A.take<uint8_t>(K);
  unsigned long long* ttot = A.take<unsigned long long>(K);
  int* tnext = A.take<int>(1);
  if (A.failed) return alloc_fail();
  const bool pre = max_triangles > 0 && E > 0 && N <= ph_triangles_total_max_vertices();
  if (pre) {
    const double bound_m = std::pow(3.0 * (double)max_triangles / std::sqrt(2.0), 2.0 / 3.0);
    const i64 m_star = std::max<i64>(0, (i64)std::floor(bound_m) - 1);  // conservative: a few more clouds counted
    count_launch();
    ph::launch_pdl(k_tri_want, dim3(grid_for(K)), dim3(256), 0, s, (const int64_t*)e_off, K, m_star, want);
    PH_TRY(ph_batch_triangles_total(adj_ptr, adj_idx, N, vcloud, want, K, ttot, tnext, s));
    count_launch();
    ph::launch_pdl(k_tri_keep, dim3(grid_for(K)), dim3(256), 0, s, (const uint8_t*)want,
                   (const unsigned long long*)ttot, K, (i64)max_triangles, tkeep);
  }
  PH_TRY(triangles_count_masked(si, sj, E, adj_ptr, adj_idx, adj_rank, tri_off, tcof_off, tc_ws, tc_b,
                                pre ? tkeep : nullptr, pre ? vcloud : nullptr, s));
  PH_TRY(ph_max_count(tcof_off, E, cnt + 8, s));  // the longest cofacet row (before any clearing: a bound)
  count_launch();
  ph::launch_pdl(k_seg_diff, dim3(grid_for(K)), dim3(256), 0, s, (const int64_t*)tri_off, (const int64_t*)e_off, K,
                 per);
  {
    Part parts[5] = {{cnt, hcnt, 16 * sizeof(int64_t)},
                     {e_off, hoff, sizeof(int64_t) * (K + 1)},
                     {per, hper, sizeof(int64_t) * K},
                     {ttot, htot, sizeof(int64_t) * K},
                     {want, hwant, (size_t)K}};
    if (readback_parts(parts, pre ? 5 : 3, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
  }
  // a cloud counted exactly and over the limit counted nothing in the per-edge pass
  if (pre)
    for (int c = 0; c < K; ++c)
      if (hwant[c] && htot[c] > max_triangles) hper[c] = htot[c];
  if ((int)(hcnt[1] >> 32) != 0) return give_up(fail((int)(hcnt[1] >> 32), "ph_boruvka_mst failed"));
  std::vector<uint8_t> keep1(K, 0), keep2(K, 0);
  i64 T = 0, span1 = 0;
  bool any_cleared = false, any_h2 = false;
  for (int c = 0; c < K; ++c) {
    res->stat[0][c] = hoff[c + 1] - hoff[c];
    res->stat[1][c] = hper[c];
    if (max_dim[c] < 1) {
      any_cleared = any_cleared || hper[c] > 0;
      continue;
    }
    if (hper[c] > max_triangles) {
      res->status[c] = PH_ERR_LIMIT;
      res->message[c] = tri_limit_msg(hper[c], max_triangles);
      any_cleared = any_cleared || hper[c] > 0;
      continue;
    }
    keep1[c] = 1;
    keep2[c] = max_dim[c] == 2;
    any_h2 = any_h2 || keep2[c];
    T += hper[c];
    span1 = std::max<i64>(span1, hper[c]);
  }
  if (E + 3 * T >= (int64_t(1) << 31) || (K > 1 && max_batch_simplices > 0 && T > max_batch_simplices)) {
    // the union's ranks do not fit int32: the caller splits the batch (the
    // per-cloud counts in the result tell it how)
    A.release_to(res->scratch);
    *out = res;
    return fail(PH_ERR_CAPACITY, "ph_rips_persistence_batch: the batch's simplices exceed the rank range or the batch budget; split it");
  }
  memcpy(hoff2, keep1.data(), K);  // staging for the flag upload (hoff2 is free until step 6)
  memcpy(reinterpret_cast<char*>(hoff2) + K, keep2.data(), K);
  if (cudaMemcpyAsync(cflag, hoff2, 2 * K, cudaMemcpyHostToDevice, s) != cudaSuccess) {
    record_error(cudaGetLastError());
    return give_up(PH_ERR_CUDA);
  }
  if (any_cleared && E) {  // no triangles for clouds over the limit or asking for H0 only
    count_launch();
    ph::launch_pdl(k_edge_flags, dim3(grid_for(E)), dim3(256), 0, s, (const i32*)si, E, (const i32*)vcloud,
                   (const uint8_t*)cflag, 0, (const uint8_t*)nullptr, eflag);
    PH_TRY(mask_offsets(A, s, tri_off, E, eflag));
    PH_TRY(mask_offsets(A, s, tcof_off, E, eflag));  // their cofacet rows go too
  }
  i32* tri_m = A.take<i32>(T);
  i32* tri_w = A.take<i32>(T);
  i32* tri_fa = A.take<i32>(T);
  i32* tri_fb = A.take<i32>(T);
  i32* off1 = A.take<i32>(E + 1);
  i32* data1 = A.take<i32>(3 * T);
  i32* cmf1 = A.take<i32>(T);
  uint8_t* skip1 = A.take<uint8_t>(E);
  int64_t* row_off1 = A.take<int64_t>(K + 1);
  int64_t* nrows1 = A.take<int64_t>(1);
  const size_t cc_b = ph_cofacet_csr_workspace_bytes(T, 3), r1_b = ph_batch_persistence_rows_workspace_bytes(E);
  void* cc_ws = A.bytes(cc_b);
  void* r1_ws = A.bytes(r1_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[1], sizeof(float) * 2 * std::max<i64>(E, 1), s) != cudaSuccess)
    return alloc_fail();
  const i64 max_row = hcnt[8];
  if (T) {
    int rc = ph_triangles_emit(si, sj, E, adj_ptr, adj_idx, adj_rank, tri_off, tri_m, tri_w, tri_fa, tri_fb, s);
    // rows scattered and sorted in shared memory when every row fits, else the radix form
    if (rc == PH_OK && max_row <= ph_cofacet_rows3_max_row()) {
      const size_t r3_b = ph_cofacet_rows3_workspace_bytes(E);
      void* r3_ws = A.bytes(r3_b);
      if (A.failed) return alloc_fail();
      rc = ph_cofacet_rows3(tri_m, tri_fa, tri_fb, T, E, (i32)E, tcof_off, (int32_t)max_row, off1, data1, st + 5,
                            r3_ws, r3_b, s);
    } else if (rc == PH_OK) {
      rc = ph_cofacet_csr(nullptr, tri_m, tri_fa, tri_fb, 3, T, E, (i32)E, off1, data1, cc_ws, cc_b, s);
    }
    if (rc == PH_OK) rc = ph_cof_max_face(nullptr, tri_m, tri_fa, tri_fb, 3, T, 0, mask, cmf1, s);
    if (rc != PH_OK) return give_up(rc);
  } else {
    ph::zero_async(off1, sizeof(i32) * (E + 1), s);
  }
  // H1 columns: the non-forest edges of the clouds kept for H1
  if (E) {
    count_launch();
    ph::launch_pdl(k_edge_flags, dim3(grid_for(E)), dim3(256), 0, s, (const i32*)si, E, (const i32*)vcloud,
                   (const uint8_t*)cflag, 1, (const uint8_t*)mask, skip1);
  }

  // ---- 5. H1 reduction and rows per cloud --------------------------------------------------------
  i64 pool1 = pool_capacity(3 * T, E);
  RedOut r1{};
  int64_t* tet_off = nullptr;
  uint8_t* en2 = nullptr;
  void* tq_ws = nullptr;
  size_t tq_b = 0;
  if (any_h2) {
    tet_off = A.take<int64_t>(E + 1);
    en2 = A.take<uint8_t>(E);
    tq_b = ph_tets_count_workspace_bytes(E);
    tq_ws = A.bytes(tq_b);
    if (A.failed) return alloc_fail();
  }
  for (int attempt = 0;; ++attempt) {
    int rc = reduce_only(A, s, off1, data1, E, 0, T, (i32)E, span1, skip1, cmf1, pool1, st + 2, r1);
    if (rc == PH_OK)
      rc = ph_batch_persistence_rows(r1.state, r1.piv, E, (i32)E, filt, nullptr, tri_m, e_off, K, res->rows[1],
                                     row_off1, nrows1, r1_ws, r1_b, s);
    if (rc != PH_OK) return give_up(rc);
    if (any_h2 && attempt == 0) {
      // tetrahedra of the clouds kept for H2, counted before waiting
      count_launch();
      ph::launch_pdl(k_edge_flags, dim3(grid_for(E)), dim3(256), 0, s, (const i32*)si, E, (const i32*)vcloud,
                     (const uint8_t*)(cflag + K), 0, (const uint8_t*)nullptr, en2);
      rc = ph_tets_count(tri_off, tri_w, E, adj_ptr, adj_idx, adj_rank, en2, tet_off, tq_ws, tq_b, s);
      if (rc == PH_OK) {
        count_launch();
        ph::launch_pdl(k_seg_diff, dim3(grid_for(K)), dim3(256), 0, s, (const int64_t*)tet_off, (const int64_t*)e_off,
                       K, per);
      }
      if (rc != PH_OK) return give_up(rc);
    }
    Part parts[3] = {{cnt, hcnt, 16 * sizeof(int64_t)},
                     {row_off1, hoff2, sizeof(int64_t) * (K + 1)},
                     {per, hper, any_h2 ? sizeof(int64_t) * K : 0}};
    if (readback_parts(parts, 3, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_red = (int)(hcnt[2] & 0xffffffff);
    if ((int)(hcnt[3] >> 32) != 0) return give_up(fail((int)(hcnt[3] >> 32), "ph_cofacet_rows3 failed"));
    if (st_red == PH_OK) break;
    if (st_red != PH_ERR_POOL || attempt >= 3 || pool1 >= POOL_MAX)
      return give_up(fail(st_red, "ph_reduce (H1) failed"));
    pool1 = std::min<i64>(pool1 * 4, POOL_MAX);
    ph::zero_async(st + 2, sizeof(int), s);
  }
  res->off[1].assign(hoff2, hoff2 + K + 1);
  if (!any_h2) {
    A.release_to(res->scratch);
    *out = res;
    return PH_OK;
  }

  // ---- 6. H2 for the clouds that ask for it -------------------------------------------------------
  i64 Q = 0, span2 = 0;
  bool any_cleared2 = false;
  for (int c = 0; c < K; ++c) {
    if (!keep2[c]) continue;
    res->stat[2][c] = hper[c];
    if (hper[c] > max_tetrahedra) {
      res->status[c] = PH_ERR_LIMIT;
      res->message[c] = tet_limit_msg(hper[c], max_tetrahedra);
      keep2[c] = 0;
      any_cleared2 = any_cleared2 || hper[c] > 0;
      continue;
    }
    Q += hper[c];
    span2 = std::max<i64>(span2, hper[c]);
  }
  if (E + T + Q >= (int64_t(1) << 31) || 4 * Q >= (int64_t(1) << 31) ||
      (K > 1 && max_batch_simplices > 0 && T + Q > max_batch_simplices)) {
    A.release_to(res->scratch);
    *out = res;
    return fail(PH_ERR_CAPACITY, "ph_rips_persistence_batch: the batch's simplices exceed the rank range or the batch budget; split it");
  }
  if (any_cleared2) {
    memcpy(hoff2, keep2.data(), K);
    if (cudaMemcpyAsync(cflag + K, hoff2, K, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      record_error(cudaGetLastError());
      return give_up(PH_ERR_CUDA);
    }
    count_launch();
    ph::launch_pdl(k_edge_flags, dim3(grid_for(E)), dim3(256), 0, s, (const i32*)si, E, (const i32*)vcloud,
                   (const uint8_t*)(cflag + K), 0, (const uint8_t*)nullptr, en2);
    PH_TRY(mask_offsets(A, s, tet_off, E, en2));
  }
  i32* tet_m = A.take<i32>(Q);
  i32* tet_faces = A.take<i32>(4 * Q);
  uint8_t* skip2 = A.take<uint8_t>(T);
  i32* cmf2 = A.take<i32>(Q);
  i32* off2 = A.take<i32>(T + 1);
  i32* data2 = A.take<i32>(4 * Q);
  int64_t* t_off = A.take<int64_t>(K + 1);
  int64_t* row_off2 = A.take<int64_t>(K + 1);
  int64_t* nrows2 = A.take<int64_t>(1);
  // the H2 cofacet rows without a global sort when every row fits the per-row
  // sorts: a triangle's tetrahedra number at most its cloud's points less 3
  i64 max_n = 0;
  for (int c = 0; c < K; ++c) max_n = std::max<i64>(max_n, segs[c].n);
  const bool rows4 = max_n - 3 <= COF_ROWS_MAX;
  const size_t c2_b = rows4 ? cofacet_rows_aos_workspace_bytes(T) : ph_cofacet_csr_workspace_bytes(Q, 4),
               r2_b = ph_batch_persistence_rows_workspace_bytes(T);
  void* c2_ws = A.bytes(c2_b);
  void* r2_ws = A.bytes(r2_b);
  if (A.failed || cudaMallocAsync((void**)&res->rows[2], sizeof(float) * 2 * std::max<i64>(T, 1), s) != cudaSuccess)
    return alloc_fail();
  {
    int rc = PH_OK;
    if (Q)
      rc = ph_tets_emit(si, sj, E, tri_off, tri_w, tri_fa, tri_fb, adj_ptr, adj_idx, adj_rank, en2, tet_off, tet_m,
                        tet_faces, st + 3, s);
    if (rc == PH_OK) rc = ph_mark_pivots(r1.state, r1.piv, E, (i32)E, skip2, T, s);
    // triangles of the clouds without H2 are not columns
    if (rc == PH_OK && T) rc = ph_or_gather_mask(skip2, en2, tri_m, T, 1, s);
    if (rc == PH_OK && Q) rc = ph_cof_max_face(tet_faces, nullptr, nullptr, nullptr, 4, Q, (i32)E, skip2, cmf2, s);
    if (rc == PH_OK && Q)
      rc = rows4 ? cofacet_rows_aos(tet_faces, 4, Q, T, (i32)(E + T), off2, data2, st + 3, c2_ws, c2_b, s)
                 : ph_cofacet_csr(tet_faces, nullptr, nullptr, nullptr, 4, Q, T, (i32)(E + T), off2, data2, c2_ws,
                                  c2_b, s);
    if (rc != PH_OK) return give_up(rc);
    if (!Q) ph::zero_async(off2, sizeof(i32) * (T + 1), s);
    count_launch();
    ph::launch_pdl(k_gather_off, dim3(grid_for(K + 1)), dim3(256), 0, s, (const int64_t*)tri_off,
                   (const int64_t*)e_off, K, t_off);
  }
  i64 pool2 = pool_capacity(4 * Q, T);
  RedOut r2{};
  for (int attempt = 0;; ++attempt) {
    int rc = reduce_only(A, s, off2, data2, T, (i32)E, Q, (i32)(E + T), span2, skip2, cmf2, pool2, st + 4, r2);
    if (rc == PH_OK)
      rc = ph_batch_persistence_rows(r2.state, r2.piv, T, (i32)(E + T), filt, tri_m, tet_m, t_off, K, res->rows[2],
                                     row_off2, nrows2, r2_ws, r2_b, s);
    if (rc != PH_OK) return give_up(rc);
    Part parts[2] = {{cnt, hcnt, 16 * sizeof(int64_t)}, {row_off2, hoff2, sizeof(int64_t) * (K + 1)}};
    if (readback_parts(parts, 2, slots, s) != PH_OK) return give_up(PH_ERR_CUDA);
    const int st_emit = (int)(hcnt[2] >> 32), st_red = (int)(hcnt[3] & 0xffffffff);
    if (st_emit) return give_up(fail(st_emit, "ph_tets_emit failed"));
    if (st_red == PH_OK) break;
    if (st_red != PH_ERR_POOL || attempt >= 3 || pool2 >= POOL_MAX)
      return give_up(fail(st_red, "ph_reduce (H2) failed"));
    pool2 = std::min<i64>(pool2 * 4, POOL_MAX);
    ph::zero_async(st + 4, sizeof(int), s);
  }
  res->off[2].assign(hoff2, hoff2 + K + 1);
  A.release_to(res->scratch);
  *out = res;
  return PH_OK;
}

extern "C" int32_t ph_batch_result_status(const ph_batch_result* r, int32_t cloud) {
  if (!r || cloud < 0 || cloud >= r->nclouds) return PH_ERR_ARG;
  return r->status[cloud];
}

extern "C" const char* ph_batch_result_message(const ph_batch_result* r, int32_t cloud) {
  if (!r || cloud < 0 || cloud >= r->nclouds) return "";
  return r->message[cloud].c_str();
}

extern "C" int64_t ph_batch_result_stat(const ph_batch_result* r, int32_t cloud, int32_t k) {
  if (!r || cloud < 0 || cloud >= r->nclouds || k < 0 || k > 2) return -1;
  return r->stat[k][cloud];
}

extern "C" int ph_batch_result_offsets(const ph_batch_result* r, int32_t dim, int64_t* out) {
  if (!r || dim < 0 || dim > 2 || !out) return PH_ERR_ARG;
  if (r->off[dim].empty()) {
    for (int c = 0; c <= r->nclouds; ++c) out[c] = 0;
    return PH_OK;
  }
  for (int c = 0; c <= r->nclouds; ++c) out[c] = r->off[dim][c];
  return PH_OK;
}

extern "C" int ph_batch_result_copy(const ph_batch_result* r, int32_t dim, float* dst, int32_t to_host,
                                    void* stream) {
  if (!r || dim < 0 || dim > 2) return PH_ERR_ARG;
  if (r->off[dim].empty() || r->off[dim].back() == 0) return PH_OK;
  if (!dst || !r->rows[dim]) return PH_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(dst, r->rows[dim], sizeof(float) * 2 * r->off[dim].back(),
                                  to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && s != r->stream) {  // frees on the run's stream wait for this copy
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      e = cudaEventRecord(ev, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(r->stream, ev, 0);
      cudaEventDestroy(ev);
    }
  }
  if (e != cudaSuccess) {
    record_error(e);
    return PH_ERR_CUDA;
  }
  return PH_OK;
}

extern "C" void ph_batch_result_free(ph_batch_result* r) {
  if (!r) return;
  for (float* p : r->rows)
    if (p) cudaFreeAsync(p, r->stream);
  for (void* p : r->scratch) cudaFreeAsync(p, r->stream);
  delete r;
}
