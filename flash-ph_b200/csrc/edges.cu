// Rips filtration on the GPU: pairwise edge enumeration, the filtration
// sort and the per-vertex adjacency.
//
// Edge enumeration (reference: kernels/edge_kernel.py:23-224) is the one
// FP32-ALU-bound stage of the pipeline: n(n-1)/2 pairs x d dimensions, two
// FP32 instructions (subtract, fused multiply-add) per pair and dimension.
// One CTA of 256 threads owns a 128 x 128 tile of the upper triangle of the
// pair matrix; both point tiles are staged in shared memory transposed
// (dimension-major, chunks of 16 dimensions) so that each thread reads its
// 8 x 8 register block with four 128-bit shared loads per dimension. The
// squared distance is accumulated in dimension order with one fused
// multiply-add per step, the arithmetic of the reference's compiled kernel.
// Hits are rare (density ~1e-4 at the benchmark sizes), so they are
// compacted with one warp-aggregated atomic on a global counter and sorted
// afterwards; the emission order does not need to be reproduced here.
#include <algorithm>
#include <cmath>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int ET = 128;  // points per tile side
constexpr int EK = 16;   // dimensions per shared-memory chunk
constexpr int ENT = 256;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void tile_coords(i64 b, i64 nt, i64& I, i64& J) {
  // b-th tile of the row-major upper triangle (I <= J) of an nt x nt grid
  const double a = 2.0 * (double)nt + 1.0;
  i64 r = (i64)floor((a - sqrt(a * a - 8.0 * (double)b)) * 0.5);
  if (r < 0) r = 0;
  auto start = [nt](i64 x) { return x * nt - x * (x - 1) / 2; };
  while (r > 0 && start(r) > b) --r;
  while (start(r + 1) <= b) ++r;
  I = r;
  J = r + (b - start(r));
}

// Finds the cloud owning work item b: the last segment with tile_off <= b.
__device__ __forceinline__ int find_seg(const ph_cloud_seg* segs, int nsegs, i64 b) {
  int lo = 0, hi = nsegs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].tile_off <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One CTA per 128 x 128 tile of one cloud's upper triangle. Single clouds
// pass their segment by value (segs == nullptr); batches pass a device table
// of ph_cloud_seg records, ordered by tile_off. Vertex indices are written
// as global indices (vbase + local).
__global__ void __launch_bounds__(ENT, 2)
    k_edges(const float* __restrict__ pts_all, const ph_cloud_seg* __restrict__ segs, int nsegs,
            ph_cloud_seg seg0, i32* __restrict__ oi, i32* __restrict__ oj, float* __restrict__ od,
            i64 cap, unsigned long long* __restrict__ count) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ __align__(16) float xs[EK][ET];
  __shared__ __align__(16) float ys[EK][ET];
  const ph_cloud_seg sg = segs ? segs[find_seg(segs, nsegs, (i64)blockIdx.x)] : seg0;
  const float* __restrict__ pts = pts_all + sg.pt_off;
  const i64 n = sg.n;
  const int d = sg.d;
  const float thr_sq = sg.thr_sq;
  const i64 nt = (n + ET - 1) / ET;
  i64 I, J;
  tile_coords((i64)blockIdx.x - sg.tile_off, nt, I, J);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const i64 i0 = I * ET, j0 = J * ET;
  float acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.0f;

  for (int k0 = 0; k0 < d; k0 += EK) {
    const int kc = min(EK, d - k0);
    const int tot = ET * kc;
    for (int idx = threadIdx.x; idx < tot; idx += ENT) {
      const int p = idx / kc, k = idx - p * kc;
      const i64 gi = i0 + p, gj = j0 + p;
      xs[k][p] = gi < n ? pts[gi * d + k0 + k] : 0.0f;
      ys[k][p] = gj < n ? pts[gj * d + k0 + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll 2
    for (int k = 0; k < kc; ++k) {
      const float4 xa = *reinterpret_cast<const float4*>(&xs[k][ty * 8]);
      const float4 xb = *reinterpret_cast<const float4*>(&xs[k][ty * 8 + 4]);
      const float4 ya = *reinterpret_cast<const float4*>(&ys[k][tx * 8]);
      const float4 yb = *reinterpret_cast<const float4*>(&ys[k][tx * 8 + 4]);
      const float xv[8] = {xa.x, xa.y, xa.z, xa.w, xb.x, xb.y, xb.z, xb.w};
      const float yv[8] = {ya.x, ya.y, ya.z, ya.w, yb.x, yb.y, yb.z, yb.w};
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float df = __fsub_rn(xv[r], yv[c]);
          acc[r][c] = __fmaf_rn(df, df, acc[r][c]);
        }
    }
    __syncthreads();
  }

  // hits of this thread's 8x8 block as a 64-bit mask
  u64 hit = 0;
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const i64 gi = i0 + ty * 8 + r, gj = j0 + tx * 8 + c;
      const bool ok = (gi < gj) && (gj < n) && (acc[r][c] < thr_sq);
      hit |= (u64)ok << (r * 8 + c);
    }
  const int cnt = __popcll(hit);
  if (!__any_sync(FULL, cnt != 0)) return;
  // warp-aggregated reservation
  const int lane = threadIdx.x & 31;
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const int wtot = __shfl_sync(FULL, incl, 31);
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(count, (unsigned long long)wtot);
  base = __shfl_sync(FULL, base, 31);
  unsigned long long pos = base + (unsigned long long)(incl - cnt);
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if ((hit >> (r * 8 + c)) & 1ull) {
        if (pos < (unsigned long long)cap) {
          oi[pos] = (i32)(sg.vbase + i0 + ty * 8 + r);
          oj[pos] = (i32)(sg.vbase + j0 + tx * 8 + c);
          od[pos] = acc[r][c];
        }
        ++pos;
      }
    }
}

// ---- filtration sort -------------------------------------------------------
__global__ void k_edge_keys(const i32* __restrict__ ei, const i32* __restrict__ ej,
                            const float* __restrict__ dsq, i64 E, u64* __restrict__ keys,
                            u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const u64 i = (u64)ei[e], j = (u64)ej[e];
    const u64 colex = j * (j - 1) / 2 + i;
    keys[e] = ((u64)float_bits(dsq[e]) << 32) | (colex & 0xffffffffull);
    vals[e] = (u32)e;
  }
}

// Position of pair (i, j), i < j, in the reference kernel's emission order:
// tiles of 32 points row-major over (I, J), row-major inside the tile.
__device__ __forceinline__ u64 emission_order(u64 i, u64 j, u64 nb32) {
  return (((i >> 5) * nb32 + (j >> 5)) << 10) | ((i & 31) << 5) | (j & 31);
}

// Runs of equal packed keys (possible only when the 32-bit colex part wraps,
// n > 92682) are put into emission order, which is what the reference's
// stable argsort of its emitted edge list produces.
__global__ void k_fix_ties(const u64* __restrict__ keys, u32* __restrict__ vals,
                           const i32* __restrict__ ei, const i32* __restrict__ ej, i64 E, u64 nb32) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < E; p += (i64)gridDim.x * blockDim.x) {
    const bool starts = (p == 0 || keys[p - 1] != keys[p]) && (p + 1 < E && keys[p + 1] == keys[p]);
    if (!starts) continue;
    i64 q = p + 1;
    while (q < E && keys[q] == keys[p]) ++q;
    for (i64 a = p + 1; a < q; ++a) {  // insertion sort of the run (runs are tiny)
      const u32 v = vals[a];
      const u64 ov = emission_order((u64)ei[v], (u64)ej[v], nb32);
      i64 b = a - 1;
      while (b >= p) {
        const u32 w = vals[b];
        if (emission_order((u64)ei[w], (u64)ej[w], nb32) <= ov) break;
        vals[b + 1] = w;
        --b;
      }
      vals[b + 1] = v;
    }
  }
}

__global__ void k_gather_edges(const u32* __restrict__ perm, const i32* __restrict__ ei,
                               const i32* __restrict__ ej, const float* __restrict__ dsq, i64 E,
                               i32* __restrict__ oi, i32* __restrict__ oj, float* __restrict__ od) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const u32 s = perm[e];
    oi[e] = ei[s];
    oj[e] = ej[s];
    od[e] = dsq[s];
  }
}

// ---- vertex CSR ---------------------------------------------------------------
// half-edge keys (vertex << sh) | neighbour, sh = the bits of a vertex index
__global__ void k_half_keys(const i32* __restrict__ ei, const i32* __restrict__ ej, i64 E, int sh,
                            u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const u64 i = (u64)(u32)ei[e], j = (u64)(u32)ej[e];
    keys[2 * e] = (i << sh) | j;
    vals[2 * e] = (u32)e;
    keys[2 * e + 1] = (j << sh) | i;
    vals[2 * e + 1] = (u32)e;
  }
}

__global__ void k_csr_fill(const u64* __restrict__ keys, const u32* __restrict__ vals, i64 H, i64 n, int sh,
                           i32* __restrict__ ptr, i32* __restrict__ idx, i32* __restrict__ rank) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const u64 low = (1ull << sh) - 1;
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < H; p += (i64)gridDim.x * blockDim.x) {
    const u64 k = keys[p];
    const i64 s = (i64)(k >> sh);
    idx[p] = (i32)(k & low);
    rank[p] = (i32)vals[p];
    const i64 prev = p ? (i64)(keys[p - 1] >> sh) : -1;
    for (i64 v = prev + 1; v <= s; ++v) ptr[v] = (i32)p;
    if (p == H - 1)
      for (i64 v = s + 1; v <= n; ++v) ptr[v] = (i32)H;
  }
}

__global__ void k_sqrt(const float* __restrict__ in, float* __restrict__ out, i64 n) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    out[i] = __fsqrt_rn(in[i]);
}

inline int grid_for(i64 n, int nt = 256) { return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16)); }

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" int ph_edges_enumerate(const float* pts, int64_t n, int32_t d, float thr_sq, int32_t* out_i,
                                  int32_t* out_j, float* out_dsq, int64_t capacity,
                                  unsigned long long* d_count, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || d <= 0 || capacity < 0 || !d_count) return PH_ERR_ARG;
  if (n >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  ph::zero_async(d_count, sizeof(unsigned long long), s);
  if (n >= 2) {
    const i64 nt = (n + ET - 1) / ET;
    const i64 tiles = nt * (nt + 1) / 2;
    if (tiles >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
    ph_cloud_seg seg{};
    seg.n = (int32_t)n;
    seg.d = d;
    seg.thr_sq = thr_sq;
    ph::count_launch();
    ph::launch_pdl(k_edges, dim3((unsigned)tiles), dim3(ENT), 0, s, pts, nullptr, 1, seg, out_i, out_j, out_dsq, capacity, d_count);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int64_t ph_cloud_tiles(int64_t n) {
  if (n < 2) return 0;
  const i64 nt = (n + ET - 1) / ET;
  return nt * (nt + 1) / 2;
}

extern "C" int ph_batch_edges_enumerate(const float* pts, const ph_cloud_seg* segs, int32_t nsegs,
                                        int64_t ntiles, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                        int64_t capacity, unsigned long long* d_count, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nsegs < 0 || ntiles < 0 || capacity < 0 || !d_count) return PH_ERR_ARG;
  if (ntiles >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  ph::zero_async(d_count, sizeof(unsigned long long), s);
  if (nsegs > 0 && ntiles > 0) {
    ph::count_launch();
    ph::launch_pdl(k_edges, dim3((unsigned)ntiles), dim3(ENT), 0, s, pts, segs, nsegs, ph_cloud_seg{}, out_i, out_j, out_dsq, capacity,
                                             d_count);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_edges_sort_workspace_bytes(int64_t E) {
  return Carve::need((size_t)E * 8) + Carve::need((size_t)E * 4) + radix_sort_workspace_bytes(E);
}

extern "C" int ph_edges_sort(const int32_t* in_i, const int32_t* in_j, const float* in_dsq, int64_t E,
                             int64_t n, int32_t* out_i, int32_t* out_j, float* out_dsq, void* workspace,
                             size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || E >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  if (E == 0) return PH_OK;
  const int rc = ph::cluster_sort_edges(in_i, in_j, in_dsq, E, n, out_i, out_j, out_dsq, s);
  if (rc != ph::CLUSTER_SORT_NA) return rc;
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(E);
  u32* vals = c.take<u32>(E);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(E));
  if (!keys || !vals || !rws) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_edge_keys, dim3(grid_for(E)), dim3(256), 0, s, in_i, in_j, in_dsq, E, keys, vals);
  PH_TRY(radix_sort_pairs(keys, vals, E, 0, 64, rws, radix_sort_workspace_bytes(E), s));
  if (n > 92682) {
    ph::count_launch();
    ph::launch_pdl(k_fix_ties, dim3(grid_for(E)), dim3(256), 0, s, keys, vals, in_i, in_j, E, (u64)((n + 31) / 32));
  }
  ph::count_launch();
  ph::launch_pdl(k_gather_edges, dim3(grid_for(E)), dim3(256), 0, s, vals, in_i, in_j, in_dsq, E, out_i, out_j, out_dsq);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_vertex_csr_workspace_bytes(int64_t E) {
  return Carve::need((size_t)E * 16) + Carve::need((size_t)E * 8) + radix_sort_workspace_bytes(2 * E);
}

extern "C" int ph_vertex_csr(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                             int32_t* adj_ptr, int32_t* adj_idx, int32_t* adj_rank, void* workspace,
                             size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || 2 * E >= (int64_t(1) << 31) || n < 0) return PH_ERR_OVERFLOW;
  if (E == 0) {
    ph::zero_async(adj_ptr, sizeof(int32_t) * (n + 1), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(2 * E);
  u32* vals = c.take<u32>(2 * E);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(2 * E));
  if (!keys || !vals || !rws) return PH_ERR_ARG;
  // sort only the key bits a vertex pair needs: 2 x bits(n - 1), in whole bytes
  int sh = 1;
  while (sh < 32 && (int64_t(1) << sh) < n) ++sh;
  const int end_bit = std::min(64, ((2 * sh + 7) / 8) * 8);
  ph::count_launch();
  ph::launch_pdl(k_half_keys, dim3(grid_for(E)), dim3(256), 0, s, edge_i, edge_j, E, sh, keys, vals);
  PH_TRY(radix_sort_pairs(keys, vals, 2 * E, 0, end_bit, rws, radix_sort_workspace_bytes(2 * E), s));
  ph::count_launch();
  ph::launch_pdl(k_csr_fill, dim3(grid_for(2 * E)), dim3(256), 0, s, keys, vals, 2 * E, n, sh, adj_ptr, adj_idx, adj_rank);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_sqrt_f32(const float* in, float* out, int64_t count, void* stream) {
  if (count < 0) return PH_ERR_ARG;
  if (count == 0) return PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_sqrt, dim3(grid_for(count)), dim3(256), 0, (cudaStream_t)stream, in, out, count);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
