// Exclusive scan and stable LSD radix sort (see prim.cuh).
#include "prim.cuh"

#include <algorithm>

namespace ph {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SCAN_NT = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_NT * SCAN_ITEMS;
constexpr int PART_NT = 1024;

// Exclusive scan of one value per thread across the block; *total gets the
// block sum. sm must hold NT/32 entries.
template <typename T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T* sm, T* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[w] = x;
  __syncthreads();
  if (w == 0) {
    T s = (lane < NT / 32) ? sm[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(FULL, s, o);
      if (lane >= o) s += y;
    }
    if (lane < NT / 32) sm[lane] = s;
  }
  __syncthreads();
  const T wp = (w > 0) ? sm[w - 1] : T(0);
  *total = sm[NT / 32 - 1];
  __syncthreads();
  return wp + x - v;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(SCAN_NT) k_scan_reduce(const In* __restrict__ in, i64 n,
                                                        Out* __restrict__ part, const int* active) {
  if (active && !*active) return;
  __shared__ Out sm[SCAN_NT / 32];
  const i64 base = (i64)blockIdx.x * SCAN_TILE;
  Out sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const i64 i = base + (i64)k * SCAN_NT + threadIdx.x;
    if (i < n) sum += (Out)in[i];
  }
  Out tot;
  block_excl_scan<Out, SCAN_NT>(sum, sm, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

template <typename Out>
__global__ void __launch_bounds__(PART_NT) k_scan_partials(Out* __restrict__ part, i64 nparts,
                                                          Out* __restrict__ out_total, const int* active) {
  if (active && !*active) return;
  __shared__ Out sm[PART_NT / 32];
  Out carry = 0;
  for (i64 b0 = 0; b0 < nparts; b0 += PART_NT) {
    const i64 i = b0 + threadIdx.x;
    const Out v = (i < nparts) ? part[i] : Out(0);
    Out tot;
    const Out ex = block_excl_scan<Out, PART_NT>(v, sm, &tot);
    if (i < nparts) part[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *out_total = carry;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(SCAN_NT) k_scan_down(const In* __restrict__ in, i64 n,
                                                      const Out* __restrict__ part,
                                                      Out* __restrict__ out, const int* active) {
  if (active && !*active) return;
  __shared__ Out sm[SCAN_NT / 32];
  __shared__ Out tile[SCAN_TILE];
  const i64 base = (i64)blockIdx.x * SCAN_TILE;
  // coalesced load into shared memory, then each thread scans 8 consecutive
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int j = k * SCAN_NT + threadIdx.x;
    const i64 i = base + j;
    tile[j] = (i < n) ? (Out)in[i] : Out(0);
  }
  __syncthreads();
  Out loc[SCAN_ITEMS];
  Out sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    loc[k] = sum;
    sum += tile[threadIdx.x * SCAN_ITEMS + k];
  }
  Out tot;
  const Out ex = block_excl_scan<Out, SCAN_NT>(sum, sm, &tot) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) tile[threadIdx.x * SCAN_ITEMS + k] = ex + loc[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int j = k * SCAN_NT + threadIdx.x;
    const i64 i = base + j;
    if (i < n) out[i] = tile[j];
  }
}

template <typename In, typename Out>
int scan_impl(const In* in, Out* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s,
              const int* active) {
  if (n < 0) return PH_ERR_ARG;
  if (n == 0) {
    cudaMemsetAsync(out, 0, sizeof(Out), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  const i64 nparts = (n + SCAN_TILE - 1) / SCAN_TILE;
  Carve c(ws, ws_bytes);
  Out* part = c.take<Out>(nparts);
  if (!part) return PH_ERR_ARG;
  ph::count_launch();
  k_scan_reduce<In, Out><<<(unsigned)nparts, SCAN_NT, 0, s>>>(in, n, part, active);
  ph::count_launch();
  k_scan_partials<Out><<<1, PART_NT, 0, s>>>(part, nparts, out + n, active);
  ph::count_launch();
  k_scan_down<In, Out><<<(unsigned)nparts, SCAN_NT, 0, s>>>(in, n, part, out, active);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

// ---------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------
constexpr int RS_NT = 256;
constexpr int RS_WARPS = RS_NT / 32;
constexpr int RS_PER_WARP = 512;
constexpr int RS_TILE = RS_WARPS * RS_PER_WARP;  // 4096 keys per block
constexpr int RS_ROUNDS = RS_PER_WARP / 32;      // 16

struct SortFlags {
  // [0..7] pass active, [8..15] active passes before this one, [16] total
  int f[24];
  unsigned long long or_bits, and_bits;
};

__global__ void k_or_and(const u64* __restrict__ keys, i64 n, SortFlags* fl) {
  u64 o = 0, a = ~0ull;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    o |= k;
    a &= k;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    o |= __shfl_xor_sync(FULL, o, d);
    a &= __shfl_xor_sync(FULL, a, d);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&fl->or_bits, (unsigned long long)o);
    atomicAnd(&fl->and_bits, (unsigned long long)a);
  }
}

__global__ void k_plan(SortFlags* fl, int begin_pass, int end_pass) {
  const u64 var = fl->or_bits ^ fl->and_bits;
  int cnt = 0;
  for (int p = 0; p < 8; ++p) {
    const int act = (p >= begin_pass && p < end_pass && ((var >> (8 * p)) & 0xffull)) ? 1 : 0;
    fl->f[p] = act;
    fl->f[8 + p] = cnt;
    cnt += act;
  }
  fl->f[16] = cnt & 1;
}

__global__ void __launch_bounds__(RS_NT) k_radix_hist(const u64* __restrict__ kA, const u64* __restrict__ kB,
                                                     i64 n, int pass, const SortFlags* fl,
                                                     u32* __restrict__ hist, int nblocks) {
  if (!fl->f[pass]) return;
  const u64* keys = (fl->f[8 + pass] & 1) ? kB : kA;
  __shared__ u32 h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int shift = 8 * pass;
  const i64 base = (i64)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int k = 0; k < RS_TILE / RS_NT; ++k) {
    const i64 i = base + (i64)k * RS_NT + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(i64)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_NT) k_radix_scatter(u64* __restrict__ kA, u32* __restrict__ vA,
                                                        u64* __restrict__ kB, u32* __restrict__ vB,
                                                        i64 n, int pass, const SortFlags* fl,
                                                        const u32* __restrict__ offs, int nblocks) {
  if (!fl->f[pass]) return;
  const bool srcB = fl->f[8 + pass] & 1;
  const u64* ks = srcB ? kB : kA;
  const u32* vs = srcB ? vB : vA;
  u64* kd = srcB ? kA : kB;
  u32* vd = srcB ? vA : vB;
  const int shift = 8 * pass;
  __shared__ u32 cnt[RS_WARPS][256];
  for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_NT) cnt[i / 256][i % 256] = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const i64 wbase = (i64)blockIdx.x * RS_TILE + (i64)w * RS_PER_WARP;
  u64 key[RS_ROUNDS];
  u32 val[RS_ROUNDS], dig[RS_ROUNDS], pos[RS_ROUNDS];
  const u32 lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    const i64 i = wbase + r * 32 + lane;
    const bool ok = i < n;
    const u64 k = ok ? ks[i] : 0ull;
    const u32 v = ok ? vs[i] : 0u;
    const u32 d = ok ? (u32)((k >> shift) & 255u) : 256u;
    const u32 peers = __match_any_sync(FULL, d);
    const u32 rank = __popc(peers & lt);
    const u32 b = (d < 256u) ? cnt[w][d] : 0u;
    __syncwarp();
    if (d < 256u && rank == 0) cnt[w][d] = b + __popc(peers);
    __syncwarp();
    key[r] = k;
    val[r] = v;
    dig[r] = d;
    pos[r] = b + rank;
  }
  __syncthreads();
  {
    u32 run = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      const u32 c = cnt[ww][threadIdx.x];
      cnt[ww][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    const u32 d = dig[r];
    if (d < 256u) {
      const u64 o = (u64)offs[(i64)d * nblocks + blockIdx.x] + cnt[w][d] + pos[r];
      kd[o] = key[r];
      vd[o] = val[r];
    }
  }
}

__global__ void k_copy_back(u64* __restrict__ kA, u32* __restrict__ vA, const u64* __restrict__ kB,
                            const u32* __restrict__ vB, i64 n, const SortFlags* fl) {
  if (!fl->f[16]) return;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    kA[i] = kB[i];
    vA[i] = vB[i];
  }
}

}  // namespace

size_t scan_workspace_bytes(i64 n) {
  const i64 nparts = (n + SCAN_TILE - 1) / SCAN_TILE + 1;
  return Carve::need((size_t)nparts * 8);
}

int scan_exclusive_i32_i32(const i32* in, i32* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s) {
  return scan_impl<i32, i32>(in, out, n, ws, ws_bytes, s, nullptr);
}
int scan_exclusive_i32_i64(const i32* in, i64* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s) {
  return scan_impl<i32, i64>(in, out, n, ws, ws_bytes, s, nullptr);
}
int scan_exclusive_u8_i32(const uint8_t* in, i32* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s) {
  return scan_impl<uint8_t, i32>(in, out, n, ws, ws_bytes, s, nullptr);
}

size_t radix_sort_workspace_bytes(i64 n) {
  const i64 nblocks = (n + RS_TILE - 1) / RS_TILE + 1;
  const i64 nh = 256 * nblocks;
  return Carve::need((size_t)n * 8) + Carve::need((size_t)n * 4) + Carve::need((size_t)(nh + 1) * 4) +
         scan_workspace_bytes(nh) + Carve::need(sizeof(SortFlags));
}

int radix_sort_pairs(u64* keys, u32* vals, i64 n, int begin_bit, int end_bit, void* ws,
                     size_t ws_bytes, cudaStream_t s) {
  if (n < 0 || n >= (i64(1) << 31) || begin_bit < 0 || end_bit > 64 || begin_bit % 8 || end_bit % 8)
    return PH_ERR_ARG;
  if (n <= 1) return PH_OK;
  const int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
  const i64 nh = (i64)256 * nblocks;
  Carve c(ws, ws_bytes);
  u64* kB = c.take<u64>(n);
  u32* vB = c.take<u32>(n);
  u32* offs = c.take<u32>(nh + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(nh));
  SortFlags* fl = c.take<SortFlags>(1);
  if (!kB || !vB || !offs || !sws || !fl) return PH_ERR_ARG;
  cudaMemsetAsync(fl, 0, sizeof(SortFlags), s);
  cudaMemsetAsync(&fl->and_bits, 0xff, sizeof(unsigned long long), s);
  const int g = (int)std::min<i64>((n + 255) / 256, 1184);
  ph::count_launch();
  k_or_and<<<g, 256, 0, s>>>(keys, n, fl);
  ph::count_launch();
  k_plan<<<1, 1, 0, s>>>(fl, begin_bit / 8, end_bit / 8);
  for (int p = begin_bit / 8; p < end_bit / 8; ++p) {
    ph::count_launch();
    k_radix_hist<<<nblocks, RS_NT, 0, s>>>(keys, kB, n, p, fl, offs, nblocks);
    PH_TRY((scan_impl<u32, u32>(offs, offs, nh, sws, scan_workspace_bytes(nh), s, &fl->f[p])));
    ph::count_launch();
    k_radix_scatter<<<nblocks, RS_NT, 0, s>>>(keys, vals, kB, vB, n, p, fl, offs, nblocks);
  }
  ph::count_launch();
  k_copy_back<<<g, 256, 0, s>>>(keys, vals, kB, vB, n, fl);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

}  // namespace ph
