// Threshold estimation kernels (reference: threshold.py:20-200).
//
// auto_threshold needs the k-th nearest-neighbour distance of every point
// and a linear-interpolation quantile of those distances; enclosing_radius
// needs min over points of the max distance to any point. Both are
// all-pairs scans with squared distances accumulated in dimension order with
// fused multiply-adds (the same arithmetic as the edge kernel). The reference
// uses torch.cdist, whose matrix-product formula rounds differently, so the
// thresholds agree within a tolerance, not bit for bit.
//
// Two forms of the k-NN scan, for a single cloud or every cloud of a batch
// (segment table; a block finds its cloud from the per-cloud offsets of
// 128-point query blocks):
//  * top list: one thread per query keeps its k <= 64 smallest squared
//    distances in a sorted list; the query block's coordinates are staged
//    dimension-major in shared memory (d up to ~200);
//  * radix select: any k, any d. A block takes 32 queries and finds each
//    query's k-th smallest squared distance bit by bit: four passes over all
//    candidates, each pass a 256-bin histogram per query (shared-memory
//    atomics) of the next 8 bits among the distances that share the bits
//    found so far. Coordinates are staged in 32-dimension chunks, so d is
//    unbounded; the four passes recompute the distances instead of storing
//    n per query.
// The reference's _tiled_knn (threshold.py:133-176) keeps a running top-k of
// cdist tiles; it clamps k to n - 1 and excludes the point itself
// (duplicates of it count, at distance 0), as both forms do.
#include <algorithm>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int KN_NT = 128;   // queries per top-list block, and per query block of the offsets
constexpr int KN_TP = 64;    // candidate points per tile (top list)
constexpr int KN_MAXK = 64;  // largest k of the top list

constexpr int KS_NT = 256;           // threads of a select / enclosing block
constexpr int KS_QB = 32;            // queries per select / enclosing block
constexpr int KS_TC = 64;            // candidates per tile
constexpr int KS_DC = 32;            // dimensions per staged chunk
constexpr int KS_R = KS_TC / (KS_NT / KS_QB);  // candidates per thread per tile (8)
constexpr int KS_SUB = KN_NT / KS_QB;          // select blocks per 128-point query block (4)

__device__ __forceinline__ int seg_of_block(const i64* __restrict__ off, int nsegs, i64 x) {
  int lo = 0, hi = nsegs - 1;  // last s with off[s] <= x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// the cloud a query block belongs to: single cloud when segs is null
struct CloudView {
  const float* pts;
  i64 n;
  int d;
  i64 qblk;     // 128-point query block within the cloud
  i64 out_off;  // output index of the cloud's first point
};

__device__ __forceinline__ CloudView cloud_view(const float* pts, i64 n, int d, const ph_cloud_seg* segs, int nsegs,
                                                const i64* qb_off, i64 block128) {
  CloudView v;
  if (!segs) {
    v.pts = pts;
    v.n = n;
    v.d = d;
    v.qblk = block128;
    v.out_off = 0;
    return v;
  }
  const int c = seg_of_block(qb_off, nsegs, block128);
  const ph_cloud_seg sg = segs[c];
  v.pts = pts + sg.pt_off;
  v.n = sg.n;
  v.d = sg.d;
  v.qblk = block128 - qb_off[c];
  v.out_off = sg.vbase;
  return v;
}

// ---- top list: k <= 64, query block staged whole -------------------------------------
__global__ void __launch_bounds__(KN_NT) k_knn_top(const float* __restrict__ pts_all, i64 n1, int d1,
                                                  const ph_cloud_seg* __restrict__ segs, int nsegs,
                                                  const i64* __restrict__ qb_off, int kreq, float* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ float sm[];
  const CloudView cv = cloud_view(pts_all, n1, d1, segs, nsegs, qb_off, blockIdx.x);
  const float* pts = cv.pts;
  const i64 n = cv.n;
  const int d = cv.d;
  const int k = (int)min((i64)kreq, n - 1);
  float* q = sm;                 // [d][KN_NT]
  float* tile = sm + d * KN_NT;  // [KN_TP][d]
  const i64 qi = cv.qblk * KN_NT + threadIdx.x;
  for (int idx = threadIdx.x; idx < d * KN_NT; idx += KN_NT) {
    const int t = idx / d, kk = idx - t * d;
    const i64 g = cv.qblk * KN_NT + t;
    q[kk * KN_NT + t] = g < n ? pts[g * d + kk] : 0.0f;
  }
  // the sorted list lives in local memory (indexed by a variable); its largest
  // entry, the only one every candidate is compared with, stays in a register
  float best[KN_MAXK];
  for (int z = 0; z < KN_MAXK; ++z) best[z] = __int_as_float(0x7f800000);
  float tau = __int_as_float(0x7f800000);
  for (i64 j0 = 0; j0 < n; j0 += KN_TP) {
    __syncthreads();
    const int tp = (int)((n - j0) < (i64)KN_TP ? (n - j0) : (i64)KN_TP);
    for (int idx = threadIdx.x; idx < tp * d; idx += KN_NT) tile[idx] = pts[j0 * d + idx];
    __syncthreads();
    if (qi >= n || k < 1) continue;
    for (int jj = 0; jj < tp; ++jj) {
      const i64 j = j0 + jj;
      float acc = 0.0f;
      for (int kk = 0; kk < d; ++kk) {
        const float df = __fsub_rn(q[kk * KN_NT + threadIdx.x], tile[jj * d + kk]);
        acc = __fmaf_rn(df, df, acc);
      }
      if (acc < tau && j != qi) {
        int z = k - 1;
        while (z > 0 && best[z - 1] > acc) {
          best[z] = best[z - 1];
          --z;
        }
        best[z] = acc;
        tau = best[k - 1];
      }
    }
  }
  if (qi < n) out[cv.out_off + qi] = k >= 1 ? __fsqrt_rn(tau) : 0.0f;
}

// ---- chunked distance tile (select and enclosing) ------------------------------------
// Thread t owns query lane ql = t % 32 and candidates cg + 8 r (r < KS_R) of
// the tile, cg = t / 32 (one value per warp, so candidate reads are
// broadcasts); acc[r] receives the squared distance accumulated over all d
// dimensions in order.
struct TileSmem {
  float qs[KS_DC][KS_QB];
  float cs[KS_TC][KS_DC + 1];
};

__device__ __forceinline__ void tile_distances(const float* __restrict__ pts, i64 n, int d, i64 q0, i64 j0,
                                               TileSmem& sh, float (&acc)[KS_R]) {
  const int t = threadIdx.x, ql = t & (KS_QB - 1), cg = t / KS_QB;
#pragma unroll
  for (int r = 0; r < KS_R; ++r) acc[r] = 0.0f;
  for (int d0 = 0; d0 < d; d0 += KS_DC) {
    const int dc = min(KS_DC, d - d0);
    __syncthreads();
    for (int idx = t; idx < KS_QB * dc; idx += KS_NT) {
      const int qq = idx / dc, kk = idx - qq * dc;
      const i64 g = q0 + qq;
      sh.qs[kk][qq] = g < n ? pts[g * d + d0 + kk] : 0.0f;
    }
    for (int idx = t; idx < KS_TC * dc; idx += KS_NT) {
      const int cc = idx / dc, kk = idx - cc * dc;
      const i64 g = j0 + cc;
      sh.cs[cc][kk] = g < n ? pts[g * d + d0 + kk] : 0.0f;
    }
    __syncthreads();
    for (int kk = 0; kk < dc; ++kk) {
      const float qv = sh.qs[kk][ql];
#pragma unroll
      for (int r = 0; r < KS_R; ++r) {
        const float df = __fsub_rn(qv, sh.cs[cg + r * (KS_NT / KS_QB)][kk]);
        acc[r] = __fmaf_rn(df, df, acc[r]);
      }
    }
  }
}

// ---- radix select: any k, any d --------------------------------------------------------
__global__ void __launch_bounds__(KS_NT) k_knn_select(const float* __restrict__ pts_all, i64 n1, int d1,
                                                     const ph_cloud_seg* __restrict__ segs, int nsegs,
                                                     const i64* __restrict__ qb_off, int kreq,
                                                     float* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ TileSmem sh;
  __shared__ u32 hist[KS_QB][256];
  __shared__ u32 prefix[KS_QB];
  __shared__ u32 rem[KS_QB];
  const CloudView cv = cloud_view(pts_all, n1, d1, segs, nsegs, qb_off, blockIdx.x / KS_SUB);
  const i64 n = cv.n;
  const int k = (int)min((i64)kreq, n - 1);
  const i64 q0 = cv.qblk * KN_NT + (i64)(blockIdx.x % KS_SUB) * KS_QB;
  if (q0 >= n) return;  // the whole block is past the cloud's end (uniform)
  const int t = threadIdx.x, ql = t & (KS_QB - 1), cg = t / KS_QB;
  const i64 qi = q0 + ql;
  if (t < KS_QB) {
    prefix[t] = 0;
    rem[t] = (u32)max(k, 1);
  }
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;  // the bits this pass decides: [shift, shift + 8)
    for (int idx = t; idx < KS_QB * 256; idx += KS_NT) (&hist[0][0])[idx] = 0;
    for (i64 j0 = 0; j0 < n; j0 += KS_TC) {
      float acc[KS_R];
      tile_distances(cv.pts, n, cv.d, q0, j0, sh, acc);  // its first barrier orders the clears above
      if (qi < n && k >= 1) {
        const u32 pre = prefix[ql];
#pragma unroll
        for (int r = 0; r < KS_R; ++r) {
          const i64 j = j0 + cg + r * (KS_NT / KS_QB);
          const u32 b = __float_as_uint(acc[r]);
          const bool same = ((u64)b >> (shift + 8)) == (u64)pre;  // pass 0: both 0
          if (j < n && j != qi && same) atomicAdd(&hist[ql][(b >> shift) & 255u], 1u);
        }
      }
    }
    __syncthreads();
    if (t < KS_QB) {  // the bin that holds the rem-th smallest among the matching values
      u32 r = rem[t], p = prefix[t];
      int b = 0;
      for (; b < 255; ++b) {
        const u32 c = hist[t][b];
        if (r <= c) break;
        r -= c;
      }
      prefix[t] = (p << 8) | (u32)b;
      rem[t] = r;
    }
    __syncthreads();
  }
  if (t < KS_QB && qi < n) out[cv.out_off + qi] = k >= 1 ? __fsqrt_rn(__uint_as_float(prefix[t])) : 0.0f;
}

// ---- enclosing radius: any d --------------------------------------------------------------
__global__ void __launch_bounds__(KS_NT) k_enclosing(const float* __restrict__ pts, i64 n, int d,
                                                    unsigned int* __restrict__ best_bits) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ TileSmem sh;
  __shared__ float red[KS_NT / KS_QB][KS_QB];
  const i64 q0 = (i64)blockIdx.x * KS_QB;
  const int t = threadIdx.x, ql = t & (KS_QB - 1), cg = t / KS_QB;
  float mx = 0.0f;
  for (i64 j0 = 0; j0 < n; j0 += KS_TC) {
    float acc[KS_R];
    tile_distances(pts, n, d, q0, j0, sh, acc);
#pragma unroll
    for (int r = 0; r < KS_R; ++r)
      if (j0 + cg + r * (KS_NT / KS_QB) < n) mx = fmaxf(mx, acc[r]);
  }
  red[cg][ql] = mx;
  __syncthreads();
  if (t < KS_QB && q0 + t < n) {
    float m = red[0][t];
    for (int g = 1; g < KS_NT / KS_QB; ++g) m = fmaxf(m, red[g][t]);
    atomicMin(best_bits, __float_as_uint(__fsqrt_rn(m)));
  }
}

// torch.quantile (linear): rank = q * (n - 1) in float32, lerp between the
// neighbouring order statistics with torch's two-sided lerp formula.
__global__ void k_quantile(const u64* __restrict__ sorted_bits, i64 n, float qf, float* out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const float rank = __fmul_rn(qf, (float)(n - 1));
  i64 lo = (i64)rank;
  const float w = __fsub_rn(rank, (float)lo);
  i64 hi = (i64)ceilf(rank);
  lo = lo < 0 ? 0 : (lo > n - 1 ? n - 1 : lo);
  hi = hi < 0 ? 0 : (hi > n - 1 ? n - 1 : hi);
  const float a = __uint_as_float((u32)(sorted_bits[lo] >> 32));
  const float b = __uint_as_float((u32)(sorted_bits[hi] >> 32));
  float r;
  if (fabsf(w) < 0.5f) r = __fadd_rn(a, __fmul_rn(w, __fsub_rn(b, a)));
  else r = __fsub_rn(b, __fmul_rn(__fsub_rn(b, a), __fsub_rn(1.0f, w)));
  *out = r;
}

__global__ void k_float_keys(const float* __restrict__ v, i64 n, u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    u32 b = __float_as_uint(v[i]);
    b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // order-preserving for all floats
    keys[i] = (u64)b << 32;
    vals[i] = (u32)i;
  }
}

__global__ void k_unflip(u64* __restrict__ keys, i64 n) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    u32 b = (u32)(keys[i] >> 32);
    b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    keys[i] = (u64)b << 32;
  }
}

__global__ void k_enclosing_init(unsigned int* bits) {
  ph::pdl_wait();
  ph::pdl_trigger();
  *bits = 0x7f800000u;  // +inf
}

__global__ void k_bits_to_float(const unsigned int* bits, float* out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  *out = __uint_as_float(*bits);
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}
inline size_t knn_top_smem(int d) { return sizeof(float) * ((size_t)d * KN_NT + (size_t)KN_TP * d); }
constexpr size_t KN_TOP_SMEM_MAX = 200 * 1024;

}  // namespace

// k-NN of a single cloud (segs null) or of every cloud of a batch: the top
// list where it applies, the radix select otherwise. nqb: 128-point query blocks.
int knn_kth_launch(const float* pts, i64 n, int d, const ph_cloud_seg* segs, int nsegs, const i64* qb_off, i64 nqb,
                   int max_d, int k, float* out, cudaStream_t s) {
  if (nqb <= 0) return PH_OK;
  const size_t smem = knn_top_smem(max_d);
  if (k <= KN_MAXK && smem <= KN_TOP_SMEM_MAX) {
    if (smem > 48 * 1024) ph::allow_dynamic_smem((const void*)k_knn_top);
    ph::count_launch();
    ph::launch_pdl(k_knn_top, dim3((unsigned)nqb), dim3(KN_NT), smem, s, pts, n, d, segs, nsegs, qb_off, k, out);
  } else {
    ph::count_launch();
    ph::launch_pdl(k_knn_select, dim3((unsigned)(nqb * KS_SUB)), dim3(KS_NT), 0, s, pts, n, d, segs, nsegs, qb_off,
                   k, out);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

}  // namespace ph

using namespace ph;

extern "C" int ph_knn_kth(const float* pts, int64_t n, int32_t d, int32_t k, float* out, void* stream) {
  if (n < 0 || d <= 0 || k < 1 || (n > 0 && k > n - 1)) return PH_ERR_ARG;
  if (n == 0) return PH_OK;
  return knn_kth_launch(pts, n, d, nullptr, 0, nullptr, (n + KN_NT - 1) / KN_NT, d, k, out, (cudaStream_t)stream);
}

extern "C" int ph_batch_knn_kth(const float* pts, const ph_cloud_seg* segs, int32_t nsegs, const int64_t* qb_off,
                                int64_t nqb, int32_t max_d, int32_t k, float* out, void* stream) {
  if (nsegs < 1 || nqb < 0 || max_d < 1 || k < 1) return PH_ERR_ARG;
  return knn_kth_launch(pts, 0, 0, segs, nsegs, qb_off, nqb, max_d, k, out, (cudaStream_t)stream);
}

extern "C" size_t ph_quantile_workspace_bytes(int64_t n) {
  return Carve::need((size_t)n * 8) + Carve::need((size_t)n * 4) + radix_sort_workspace_bytes(n);
}

extern "C" int ph_quantile_f32(const float* values, int64_t n, double q, float* d_out, void* workspace,
                               size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n <= 0 || !(q >= 0.0 && q <= 1.0)) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(n);
  u32* vals = c.take<u32>(n);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(n));
  if (!keys || !vals || !rws) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_float_keys, dim3(grid_for(n)), dim3(256), 0, s, values, n, keys, vals);
  PH_TRY(radix_sort_pairs(keys, vals, n, 32, 64, rws, radix_sort_workspace_bytes(n), s));
  ph::count_launch();
  ph::launch_pdl(k_unflip, dim3(grid_for(n)), dim3(256), 0, s, keys, n);
  ph::count_launch();
  ph::launch_pdl(k_quantile, dim3(1), dim3(1), 0, s, keys, n, (float)q, d_out);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_enclosing_radius_workspace_bytes(int64_t n) {
  (void)n;
  return Carve::need(sizeof(unsigned int));
}

extern "C" int ph_enclosing_radius(const float* pts, int64_t n, int32_t d, float* d_out, void* workspace,
                                   size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n <= 0 || d <= 0) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  unsigned int* bits = c.take<unsigned int>(1);
  if (!bits) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_enclosing_init, dim3(1), dim3(1), 0, s, bits);
  ph::count_launch();
  ph::launch_pdl(k_enclosing, dim3((unsigned)((n + KS_QB - 1) / KS_QB)), dim3(KS_NT), 0, s, pts, n, d, bits);
  ph::count_launch();
  ph::launch_pdl(k_bits_to_float, dim3(1), dim3(1), 0, s, bits, d_out);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
