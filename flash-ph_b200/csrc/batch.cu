// Batches of point clouds (the batching and serving forms) and the row
// assembly shared with the single-cloud path.
//
// A batch is the disjoint union of its clouds: vertex v of cloud c has the
// global index vbase_c + v. Adjacency, forest, triangles, tetrahedra and the
// reduction run on global indices unchanged. What needs the cloud structure:
//   - the filtration order is per cloud: edges are sorted by the reference's
//     packed key with local indices, then stably by cloud, so every cloud's
//     edges are contiguous and in its own filtration order;
//   - H0 and H1/H2 rows are assembled per cloud.
// Row assembly needs no sort: columns in index order have non-decreasing
// birth values (edges by rank, triangles by largest edge), so the reference's
// stable sort by birth of [apparent pairs ascending, residual pairs
// descending, essential columns descending] (reduce_h1_gpu.py:574-604) only
// reorders runs of equal birth value. Each run is ordered locally and written
// at its exclusive-scan position.
#include <algorithm>

#include "prim.cuh"

namespace ph {
namespace {

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}

__device__ __forceinline__ int seg_of(const i64* __restrict__ off, int nsegs, i64 x) {
  // last s with off[s] <= x
  int lo = 0, hi = nsegs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_vertex_cloud(const ph_cloud_seg* __restrict__ segs, int nsegs, i32* __restrict__ vcloud) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x; c < nsegs; c += gridDim.x)
    for (i64 v = threadIdx.x; v < segs[c].n; v += blockDim.x) vcloud[segs[c].vbase + v] = c;
}

// ---- per-cloud filtration sort ------------------------------------------------
__global__ void k_local_keys(const i32* __restrict__ ei, const i32* __restrict__ ej, const float* __restrict__ dsq,
                             i64 E, const i32* __restrict__ vcloud, const ph_cloud_seg* __restrict__ segs,
                             u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const i32 c = vcloud[ei[e]];
    const u64 vb = (u64)segs[c].vbase;
    const u64 i = (u64)ei[e] - vb, j = (u64)ej[e] - vb;
    const u64 colex = j * (j - 1) / 2 + i;
    keys[e] = ((u64)float_bits(dsq[e]) << 32) | (colex & 0xffffffffull);
    vals[e] = (u32)e;
  }
}

__global__ void k_cloud_keys(const u32* __restrict__ perm, const i32* __restrict__ ei, i64 E,
                             const i32* __restrict__ vcloud, u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x; k < E; k += (i64)gridDim.x * blockDim.x) {
    const u32 e = perm[k];
    keys[k] = (u64)(u32)vcloud[ei[e]];
    vals[k] = e;
  }
}

__device__ __forceinline__ u64 packed_key(u32 e, const i32* ei, const i32* ej, const float* dsq,
                                          const i32* vcloud, const ph_cloud_seg* segs) {
  const i32 c = vcloud[ei[e]];
  const u64 vb = (u64)segs[c].vbase;
  const u64 i = (u64)ei[e] - vb, j = (u64)ej[e] - vb;
  return ((u64)float_bits(dsq[e]) << 32) | ((j * (j - 1) / 2 + i) & 0xffffffffull);
}

__device__ __forceinline__ u64 emission_order_local(u32 e, const i32* ei, const i32* ej, const i32* vcloud,
                                                    const ph_cloud_seg* segs) {
  const i32 c = vcloud[ei[e]];
  const u64 vb = (u64)segs[c].vbase;
  const u64 i = (u64)ei[e] - vb, j = (u64)ej[e] - vb;
  const u64 nb32 = ((u64)segs[c].n + 31) / 32;
  return (((i >> 5) * nb32 + (j >> 5)) << 10) | ((i & 31) << 5) | (j & 31);
}

// Equal packed keys within a cloud (only when its colex part wraps) are put
// into the reference kernel's emission order.
__global__ void k_fix_ties_batch(u32* __restrict__ vals, i64 E, const i32* __restrict__ ei,
                                 const i32* __restrict__ ej, const float* __restrict__ dsq,
                                 const i32* __restrict__ vcloud, const ph_cloud_seg* __restrict__ segs) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < E; p += (i64)gridDim.x * blockDim.x) {
    const u32 ep = vals[p];
    const i32 cp = vcloud[ei[ep]];
    if (segs[cp].n <= 92682) continue;
    const u64 kp = packed_key(ep, ei, ej, dsq, vcloud, segs);
    if (p > 0) {
      const u32 eq = vals[p - 1];
      if (vcloud[ei[eq]] == cp && packed_key(eq, ei, ej, dsq, vcloud, segs) == kp) continue;
    }
    i64 q = p + 1;
    while (q < E && vcloud[ei[vals[q]]] == cp && packed_key(vals[q], ei, ej, dsq, vcloud, segs) == kp) ++q;
    for (i64 a = p + 1; a < q; ++a) {
      const u32 v = vals[a];
      const u64 ov = emission_order_local(v, ei, ej, vcloud, segs);
      i64 b = a - 1;
      while (b >= p && emission_order_local(vals[b], ei, ej, vcloud, segs) > ov) {
        vals[b + 1] = vals[b];
        --b;
      }
      vals[b + 1] = v;
    }
  }
}

__global__ void k_gather3(const u32* __restrict__ perm, const i32* __restrict__ ei, const i32* __restrict__ ej,
                          const float* __restrict__ dsq, i64 E, i32* __restrict__ oi, i32* __restrict__ oj,
                          float* __restrict__ od) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const u32 s = perm[e];
    oi[e] = ei[s];
    oj[e] = ej[s];
    od[e] = dsq[s];
  }
}

// off[c] = first item of cloud c (items grouped by cloud), off[nsegs] = n.
__global__ void k_item_offsets(const i32* __restrict__ item_vertex, i64 n, const i32* __restrict__ vcloud,
                               int nsegs, i64* __restrict__ off) {
  ph::pdl_wait();
  ph::pdl_trigger();
  if (n == 0) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= nsegs; c += gridDim.x * blockDim.x) off[c] = 0;
    return;
  }
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (i64)gridDim.x * blockDim.x) {
    const int c = vcloud[item_vertex[p]];
    const int prev = p ? vcloud[item_vertex[p - 1]] : -1;
    for (int s = prev + 1; s <= c; ++s) off[s] = p;
    if (p == n - 1)
      for (int s = c + 1; s <= nsegs; ++s) off[s] = n;
  }
}

// ---- H0 rows per cloud ---------------------------------------------------------
__global__ void k_h0_batch_edges(const float* __restrict__ filt, const uint8_t* __restrict__ mst,
                                 const i32* __restrict__ pos, i64 E, const i64* __restrict__ eoff, int nsegs,
                                 const ph_cloud_seg* __restrict__ segs, float* __restrict__ rows) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    if (!mst[e]) continue;
    const int c = seg_of(eoff, nsegs, e);
    const i64 r = segs[c].vbase + (pos[e] - pos[eoff[c]]);
    rows[2 * r] = 0.0f;
    rows[2 * r + 1] = filt[e];
  }
}

__global__ void k_h0_batch_inf(const i32* __restrict__ pos, const i64* __restrict__ eoff, int nsegs,
                               const ph_cloud_seg* __restrict__ segs, const i32* __restrict__ vcloud, i64 N,
                               float* __restrict__ rows) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (i64)gridDim.x * blockDim.x) {
    const int c = vcloud[r];
    const i64 k = r - segs[c].vbase;
    const i64 nm = pos[eoff[c + 1]] - pos[eoff[c]];
    if (k >= nm) {
      rows[2 * r] = 0.0f;
      rows[2 * r + 1] = __int_as_float(0x7f800000);
    }
  }
}

// ---- persistence rows without a sort -------------------------------------------
__device__ __forceinline__ float col_birth(i64 c, const float* filt, const i32* col_m) {
  return filt[col_m ? col_m[c] : (i32)c];
}

__device__ __forceinline__ bool row_kept(i64 c, const i32* state, const i32* piv, i32 row_base, const float* filt,
                                         const i32* col_m, const i32* row_m) {
  const i32 st = state[c];
  if (st == 3) return true;
  if (st != 1 && st != 2) return false;
  return filt[row_m[piv[c] - row_base]] > col_birth(c, filt, col_m);
}

__global__ void k_rows_flags(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                             const float* __restrict__ filt, const i32* __restrict__ col_m,
                             const i32* __restrict__ row_m, uint8_t* __restrict__ kept) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x)
    kept[c] = row_kept(c, state, piv, row_base, filt, col_m, row_m) ? 1 : 0;
}

__device__ __forceinline__ void write_row(i64 at, i64 c, const i32* state, const i32* piv, i32 row_base,
                                          const float* filt, const i32* col_m, const i32* row_m, float* rows) {
  rows[2 * at] = col_birth(c, filt, col_m);
  rows[2 * at + 1] = state[c] == 3 ? __int_as_float(0x7f800000) : filt[row_m[piv[c] - row_base]];
}

__global__ void k_rows_write(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                             const float* __restrict__ filt, const i32* __restrict__ col_m,
                             const i32* __restrict__ row_m, const uint8_t* __restrict__ kept,
                             const i32* __restrict__ pos, const i64* __restrict__ col_off, int nsegs,
                             float* __restrict__ rows) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x) {
    const int s = col_off ? seg_of(col_off, nsegs, c) : 0;
    const i64 s0 = col_off ? col_off[s] : 0, s1 = col_off ? col_off[s + 1] : K;
    const u32 b = float_bits(col_birth(c, filt, col_m));
    if (c > s0 && float_bits(col_birth(c - 1, filt, col_m)) == b) continue;  // not the start of its run
    i64 g = c + 1;
    while (g < s1 && float_bits(col_birth(g, filt, col_m)) == b) ++g;
    if (g == c + 1) {
      if (kept[c]) write_row(pos[c], c, state, piv, row_base, filt, col_m, row_m, rows);
      continue;
    }
    i64 at = pos[c];
    for (i64 x = c; x < g; ++x)  // apparent pairs, ascending column
      if (kept[x] && state[x] == 1) write_row(at++, x, state, piv, row_base, filt, col_m, row_m, rows);
    for (i64 x = g - 1; x >= c; --x)  // reduced pairs, descending column
      if (kept[x] && state[x] == 2) write_row(at++, x, state, piv, row_base, filt, col_m, row_m, rows);
    for (i64 x = g - 1; x >= c; --x)  // essential columns, descending column
      if (kept[x] && state[x] == 3) write_row(at++, x, state, piv, row_base, filt, col_m, row_m, rows);
  }
}

__global__ void k_rows_offsets(const i32* __restrict__ pos, i64 K, const i64* __restrict__ col_off, int nsegs,
                               i64* __restrict__ row_off, i64* __restrict__ d_nrows) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= nsegs; s += gridDim.x * blockDim.x)
    if (row_off) row_off[s] = pos[col_off ? col_off[s] : (s ? K : 0)];
  if (blockIdx.x == 0 && threadIdx.x == 0 && d_nrows) *d_nrows = pos[K];
}

// ---- masks -----------------------------------------------------------------------
__global__ void k_edge_dim_mask(const i32* __restrict__ ei, i64 E, const i32* __restrict__ vcloud,
                                const ph_cloud_seg* __restrict__ segs, int min_dim, uint8_t* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x)
    out[e] = segs[vcloud[ei[e]]].max_dim >= min_dim ? 1 : 0;
}

__global__ void k_or_gather(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, const i32* __restrict__ idx,
                            i64 n, int invert) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const uint8_t v = src[idx[i]];
    dst[i] |= invert ? (uint8_t)!v : v;
  }
}

// ---- thresholds per cloud (the k-NN scan is in threshold.cu) ----------------------------
__global__ void k_seg_value_keys(const float* __restrict__ v, i64 N, const i32* __restrict__ vcloud,
                                 u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (i64)gridDim.x * blockDim.x) {
    u32 b = __float_as_uint(v[i]);
    b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    keys[i] = ((u64)(u32)vcloud[i] << 32) | b;
    vals[i] = (u32)i;
  }
}

__device__ __forceinline__ float unflip(u64 key) {
  u32 b = (u32)(key & 0xffffffffull);
  b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
  return __uint_as_float(b);
}

// torch.quantile (linear) per cloud on the cloud's sorted values.
__global__ void k_seg_quantile(const u64* __restrict__ sorted, const ph_cloud_seg* __restrict__ segs, int nsegs,
                               float qf, float* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nsegs; c += gridDim.x * blockDim.x) {
    const i64 n = segs[c].n;
    if (n <= 1) {
      out[c] = 0.0f;
      continue;
    }
    const u64* s = sorted + segs[c].vbase;
    const float rank = __fmul_rn(qf, (float)(n - 1));
    i64 lo = (i64)rank;
    const float w = __fsub_rn(rank, (float)lo);
    i64 hi = (i64)ceilf(rank);
    lo = lo < 0 ? 0 : (lo > n - 1 ? n - 1 : lo);
    hi = hi < 0 ? 0 : (hi > n - 1 ? n - 1 : hi);
    const float a = unflip(s[lo]), b = unflip(s[hi]);
    out[c] = fabsf(w) < 0.5f ? __fadd_rn(a, __fmul_rn(w, __fsub_rn(b, a)))
                             : __fsub_rn(b, __fmul_rn(__fsub_rn(b, a), __fsub_rn(1.0f, w)));
  }
}

}  // namespace

// Internal: row assembly for one or more column segments.
int rows_nosort(const i32* state, const i32* piv, i64 K, i32 row_base, const float* filt, const i32* col_m,
                const i32* row_m, const i64* col_off, int nsegs, float* out_rows, i64* row_off, i64* d_nrows,
                void* ws, size_t ws_bytes, cudaStream_t s) {
  Carve c(ws, ws_bytes);
  uint8_t* kept = c.take<uint8_t>(std::max<i64>(K, 1));
  i32* pos = c.take<i32>(K + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(K));
  if (!kept || !pos || !sws) return PH_ERR_ARG;
  if (K > 0) {
    ph::count_launch();
    ph::launch_pdl(k_rows_flags, dim3(grid_for(K)), dim3(256), 0, s, state, piv, K, row_base, filt, col_m, row_m, kept);
  }
  PH_TRY(scan_exclusive_u8_i32(kept, pos, K, sws, scan_workspace_bytes(K), s));
  if (K > 0) {
    ph::count_launch();
    ph::launch_pdl(k_rows_write, dim3(grid_for(K)), dim3(256), 0, s, state, piv, K, row_base, filt, col_m, row_m, kept, pos, col_off,
                                             nsegs, out_rows);
  }
  ph::count_launch();
  ph::launch_pdl(k_rows_offsets, dim3(1), dim3(256), 0, s, pos, K, col_off, nsegs, row_off, d_nrows);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

size_t rows_nosort_workspace_bytes(i64 K) {
  return Carve::need((size_t)std::max<i64>(K, 1)) + Carve::need((size_t)(K + 1) * 4) + scan_workspace_bytes(K);
}

}  // namespace ph

using namespace ph;

extern "C" int ph_batch_vertex_cloud(const ph_cloud_seg* segs, int32_t nsegs, int32_t* vcloud, void* stream) {
  if (nsegs < 0) return PH_ERR_ARG;
  if (nsegs == 0) return PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_vertex_cloud, dim3(std::min(nsegs, 4096)), dim3(256), 0, (cudaStream_t)stream, segs, nsegs, vcloud);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_batch_edges_sort_workspace_bytes(int64_t E) {
  return 2 * Carve::need((size_t)E * 8) + 2 * Carve::need((size_t)E * 4) + radix_sort_workspace_bytes(E);
}

extern "C" int ph_batch_edges_sort(const int32_t* in_i, const int32_t* in_j, const float* in_dsq, int64_t E,
                                   const int32_t* vcloud, const ph_cloud_seg* segs, int32_t nsegs,
                                   int32_t any_wrap, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || E >= (int64_t(1) << 31) || nsegs < 1) return E < 0 ? PH_ERR_ARG : (nsegs < 1 ? PH_ERR_ARG : PH_ERR_OVERFLOW);
  if (E == 0) return PH_OK;
  Carve c(workspace, workspace_bytes);
  u64* k1 = c.take<u64>(E);
  u32* v1 = c.take<u32>(E);
  u64* k2 = c.take<u64>(E);
  u32* v2 = c.take<u32>(E);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(E));
  if (!k1 || !v1 || !k2 || !v2 || !rws) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_local_keys, dim3(grid_for(E)), dim3(256), 0, s, in_i, in_j, in_dsq, E, vcloud, segs, k1, v1);
  PH_TRY(radix_sort_pairs(k1, v1, E, 0, 64, rws, radix_sort_workspace_bytes(E), s));
  ph::count_launch();
  ph::launch_pdl(k_cloud_keys, dim3(grid_for(E)), dim3(256), 0, s, v1, in_i, E, vcloud, k2, v2);
  PH_TRY(radix_sort_pairs(k2, v2, E, 0, 32, rws, radix_sort_workspace_bytes(E), s));
  if (any_wrap) {
    ph::count_launch();
    ph::launch_pdl(k_fix_ties_batch, dim3(grid_for(E)), dim3(256), 0, s, v2, E, in_i, in_j, in_dsq, vcloud, segs);
  }
  ph::count_launch();
  ph::launch_pdl(k_gather3, dim3(grid_for(E)), dim3(256), 0, s, v2, in_i, in_j, in_dsq, E, out_i, out_j, out_dsq);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_batch_item_offsets(const int32_t* item_vertex, int64_t n_items, const int32_t* vcloud,
                                     int32_t nsegs, int64_t* off, void* stream) {
  if (n_items < 0 || nsegs < 1) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_item_offsets, dim3(grid_for(std::max<i64>(n_items, nsegs + 1))), dim3(256), 0, (cudaStream_t)stream, 
      item_vertex, n_items, vcloud, nsegs, off);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_batch_h0_rows_workspace_bytes(int64_t E) {
  return Carve::need((size_t)(E + 1) * 4) + scan_workspace_bytes(E);
}

extern "C" int ph_batch_h0_rows(const float* edge_filt, const uint8_t* mst_mask, int64_t E, const int64_t* edge_off,
                                const ph_cloud_seg* segs, int32_t nsegs, const int32_t* vcloud, int64_t N,
                                float* out_rows, void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || N < 0 || nsegs < 1) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  i32* pos = c.take<i32>(E + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(E));
  if (!pos || !sws) return PH_ERR_ARG;
  PH_TRY(scan_exclusive_u8_i32(mst_mask, pos, E, sws, scan_workspace_bytes(E), s));
  if (E > 0) {
    ph::count_launch();
    ph::launch_pdl(k_h0_batch_edges, dim3(grid_for(E)), dim3(256), 0, s, edge_filt, mst_mask, pos, E, edge_off, nsegs, segs, out_rows);
  }
  if (N > 0) {
    ph::count_launch();
    ph::launch_pdl(k_h0_batch_inf, dim3(grid_for(N)), dim3(256), 0, s, pos, edge_off, nsegs, segs, vcloud, N, out_rows);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_batch_persistence_rows_workspace_bytes(int64_t K) { return rows_nosort_workspace_bytes(K); }

extern "C" int ph_batch_persistence_rows(const int32_t* col_state, const int32_t* col_piv, int64_t K,
                                         int32_t row_base, const float* filt, const int32_t* col_m,
                                         const int32_t* row_m, const int64_t* col_off, int32_t nsegs,
                                         float* out_rows, int64_t* row_off, int64_t* d_nrows, void* workspace,
                                         size_t workspace_bytes, void* stream) {
  if (K < 0 || nsegs < 1 || (nsegs > 1 && !col_off)) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  return rows_nosort(col_state, col_piv, K, row_base, filt, col_m, row_m, col_off, nsegs, out_rows, row_off,
                     d_nrows, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int ph_batch_edge_dim_mask(const int32_t* edge_i, int64_t E, const int32_t* vcloud,
                                      const ph_cloud_seg* segs, int32_t min_dim, uint8_t* out, void* stream) {
  if (E < 0) return PH_ERR_ARG;
  if (E == 0) return PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_edge_dim_mask, dim3(grid_for(E)), dim3(256), 0, (cudaStream_t)stream, edge_i, E, vcloud, segs, min_dim, out);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_or_gather_mask(uint8_t* dst, const uint8_t* src, const int32_t* idx, int64_t n, int32_t invert,
                                 void* stream) {
  if (n < 0) return PH_ERR_ARG;
  if (n == 0) return PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_or_gather, dim3(grid_for(n)), dim3(256), 0, (cudaStream_t)stream, dst, src, idx, n, invert);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_batch_quantile_workspace_bytes(int64_t N) {
  return Carve::need((size_t)N * 8) + Carve::need((size_t)N * 4) + radix_sort_workspace_bytes(N);
}

extern "C" int ph_batch_quantile(const float* values, int64_t N, const int32_t* vcloud, const ph_cloud_seg* segs,
                                 int32_t nsegs, double q, float* out, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (N < 0 || nsegs < 1 || !(q >= 0.0 && q <= 1.0)) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(std::max<i64>(N, 1));
  u32* vals = c.take<u32>(std::max<i64>(N, 1));
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(N));
  if (!keys || !vals || !rws) return PH_ERR_ARG;
  if (N > 0) {
    ph::count_launch();
    ph::launch_pdl(k_seg_value_keys, dim3(grid_for(N)), dim3(256), 0, s, values, N, vcloud, keys, vals);
    PH_TRY(radix_sort_pairs(keys, vals, N, 0, 64, rws, radix_sort_workspace_bytes(N), s));
  }
  ph::count_launch();
  ph::launch_pdl(k_seg_quantile, dim3(grid_for(nsegs)), dim3(256), 0, s, keys, segs, nsegs, (float)q, out);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
