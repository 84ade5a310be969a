// Threshold estimation kernels (reference: threshold.py:20-200).
//
// auto_threshold needs the k-th nearest-neighbour distance of every point
// and a linear-interpolation quantile of those distances; enclosing_radius
// needs min over points of the max distance to any point. Both are
// all-pairs scans: one thread per query point, the query block's
// coordinates staged dimension-major in shared memory, candidate points
// streamed through shared memory in tiles, squared distances accumulated in
// dimension order with fused multiply-adds (the same arithmetic as the edge
// kernel). The reference uses torch.cdist, whose matrix-product formula
// rounds differently, so thresholds agree within a tolerance, not bit for bit.
#include <algorithm>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int KN_NT = 128;
constexpr int KN_TP = 64;   // candidate points per tile
constexpr int KN_MAXK = 64;

__global__ void __launch_bounds__(KN_NT) k_knn(const float* __restrict__ pts, i64 n, int d, int k,
                                              float* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ float sm[];
  float* q = sm;                 // [d][KN_NT]
  float* tile = sm + d * KN_NT;  // [KN_TP][d]
  const i64 qi = (i64)blockIdx.x * KN_NT + threadIdx.x;
  for (int idx = threadIdx.x; idx < d * KN_NT; idx += KN_NT) {
    const int t = idx / d, kk = idx - t * d;
    const i64 g = (i64)blockIdx.x * KN_NT + t;
    q[kk * KN_NT + t] = g < n ? pts[g * d + kk] : 0.0f;
  }
  float best[KN_MAXK];
  for (int z = 0; z < KN_MAXK; ++z) best[z] = __int_as_float(0x7f800000);
  for (i64 j0 = 0; j0 < n; j0 += KN_TP) {
    __syncthreads();
    const int tp = (int)((n - j0) < (i64)KN_TP ? (n - j0) : (i64)KN_TP);
    for (int idx = threadIdx.x; idx < tp * d; idx += KN_NT) tile[idx] = pts[j0 * d + idx];
    __syncthreads();
    if (qi >= n) continue;
    for (int jj = 0; jj < tp; ++jj) {
      const i64 j = j0 + jj;
      float acc = 0.0f;
      for (int kk = 0; kk < d; ++kk) {
        const float df = __fsub_rn(q[kk * KN_NT + threadIdx.x], tile[jj * d + kk]);
        acc = __fmaf_rn(df, df, acc);
      }
      if (j != qi && acc < best[k - 1]) {
        int z = k - 1;
        while (z > 0 && best[z - 1] > acc) {
          best[z] = best[z - 1];
          --z;
        }
        best[z] = acc;
      }
    }
  }
  if (qi < n) out[qi] = __fsqrt_rn(best[k - 1]);
}

__global__ void __launch_bounds__(KN_NT) k_enclosing(const float* __restrict__ pts, i64 n, int d,
                                                    unsigned int* __restrict__ best_bits) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ float sm[];
  float* q = sm;
  float* tile = sm + d * KN_NT;
  const i64 qi = (i64)blockIdx.x * KN_NT + threadIdx.x;
  for (int idx = threadIdx.x; idx < d * KN_NT; idx += KN_NT) {
    const int t = idx / d, kk = idx - t * d;
    const i64 g = (i64)blockIdx.x * KN_NT + t;
    q[kk * KN_NT + t] = g < n ? pts[g * d + kk] : 0.0f;
  }
  float mx = 0.0f;
  for (i64 j0 = 0; j0 < n; j0 += KN_TP) {
    __syncthreads();
    const int tp = (int)((n - j0) < (i64)KN_TP ? (n - j0) : (i64)KN_TP);
    for (int idx = threadIdx.x; idx < tp * d; idx += KN_NT) tile[idx] = pts[j0 * d + idx];
    __syncthreads();
    if (qi >= n) continue;
    for (int jj = 0; jj < tp; ++jj) {
      float acc = 0.0f;
      for (int kk = 0; kk < d; ++kk) {
        const float df = __fsub_rn(q[kk * KN_NT + threadIdx.x], tile[jj * d + kk]);
        acc = __fmaf_rn(df, df, acc);
      }
      mx = fmaxf(mx, acc);
    }
  }
  if (qi < n) atomicMin(best_bits, __float_as_uint(__fsqrt_rn(mx)));
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

__global__ void k_bits_to_float(const unsigned int* bits, float* out) {
  ph::pdl_wait();
  ph::pdl_trigger(); *out = __uint_as_float(*bits); }

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}
inline size_t knn_smem(int d) { return sizeof(float) * ((size_t)d * KN_NT + (size_t)KN_TP * d); }

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" int ph_knn_kth(const float* pts, int64_t n, int32_t d, int32_t k, float* out, void* stream) {
  if (n < 0 || d <= 0 || k < 1 || k > KN_MAXK || (n > 0 && k > n - 1)) return PH_ERR_ARG;
  if (n == 0) return PH_OK;
  const size_t smem = knn_smem(d);
  if (smem > 200 * 1024) return PH_ERR_ARG;
  if (smem > 48 * 1024) ph::allow_dynamic_smem((const void*)k_knn);
  ph::count_launch();
  ph::launch_pdl(k_knn, dim3((unsigned)((n + KN_NT - 1) / KN_NT)), dim3(KN_NT), smem, (cudaStream_t)stream, pts, n, d, k, out);
  PH_CHECK_LAUNCH();
  return PH_OK;
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
  const size_t smem = knn_smem(d);
  if (smem > 200 * 1024) return PH_ERR_ARG;
  if (smem > 48 * 1024) ph::allow_dynamic_smem((const void*)k_enclosing);
  cudaMemsetAsync(bits, 0x7f, sizeof(unsigned int), s);
  ph::count_launch();
  ph::launch_pdl(k_enclosing, dim3((unsigned)((n + KN_NT - 1) / KN_NT)), dim3(KN_NT), smem, s, pts, n, d, bits);
  ph::count_launch();
  ph::launch_pdl(k_bits_to_float, dim3(1), dim3(1), 0, s, bits, d_out);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
