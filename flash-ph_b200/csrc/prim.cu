// Exclusive scan and stable LSD radix sort (see prim.cuh).
#include "prim.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>
#include <type_traits>

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
  ph::pdl_wait();
  ph::pdl_trigger();
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
  ph::pdl_wait();
  ph::pdl_trigger();
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
  ph::pdl_wait();
  ph::pdl_trigger();
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

// Single-launch form for scans of up to COOP_MAX_PARTS tiles: every block
// sums its tiles, a grid barrier, then every block scans the tile sums in
// shared memory and writes its tiles (one launch instead of three, and no
// state that needs clearing beforehand).
constexpr int COOP_MAX_PARTS = 2048;

template <typename In, typename Out>
__global__ void __launch_bounds__(SCAN_NT) k_scan_coop(const In* __restrict__ in, i64 n, i64 nparts,
                                                      Out* __restrict__ part, Out* __restrict__ out,
                                                      const int* active) {
  ph::pdl_wait();
  ph::pdl_trigger();
  if (active && !*active) return;  // the flag is the same for every block
  __shared__ Out sm[SCAN_NT / 32];
  __shared__ Out spre[COOP_MAX_PARTS];
  __shared__ Out tile[SCAN_TILE];
  cooperative_groups::grid_group g = cooperative_groups::this_grid();
  for (i64 t = blockIdx.x; t < nparts; t += gridDim.x) {
    const i64 base = t * SCAN_TILE;
    Out sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const i64 i = base + (i64)k * SCAN_NT + threadIdx.x;
      if (i < n) sum += (Out)in[i];
    }
    Out tot;
    block_excl_scan<Out, SCAN_NT>(sum, sm, &tot);
    if (threadIdx.x == 0) part[t] = tot;
  }
  g.sync();
  // exclusive scan of all tile sums into shared memory
  Out carry = 0;
  for (i64 b0 = 0; b0 < nparts; b0 += SCAN_NT) {
    const i64 i = b0 + threadIdx.x;
    const Out v = i < nparts ? __ldcg(part + i) : Out(0);
    Out tot;
    const Out ex = block_excl_scan<Out, SCAN_NT>(v, sm, &tot);
    if (i < nparts) spre[i] = carry + ex;
    carry += tot;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = carry;
  __syncthreads();
  for (i64 t = blockIdx.x; t < nparts; t += gridDim.x) {
    const i64 base = t * SCAN_TILE;
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
    const Out ex = block_excl_scan<Out, SCAN_NT>(sum, sm, &tot) + spre[t];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) tile[threadIdx.x * SCAN_ITEMS + k] = ex + loc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      const int j = k * SCAN_NT + threadIdx.x;
      const i64 i = base + j;
      if (i < n) out[i] = tile[j];
    }
    __syncthreads();
  }
}

template <typename In, typename Out>
int scan_impl(const In* in, Out* out, i64 n, void* ws, size_t ws_bytes, cudaStream_t s,
              const int* active) {
  if (n < 0) return PH_ERR_ARG;
  if (n == 0) {
    ph::zero_async(out, sizeof(Out), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  const i64 nparts = (n + SCAN_TILE - 1) / SCAN_TILE;
  Carve c(ws, ws_bytes);
  Out* part = c.take<Out>(nparts);
  if (!part) return PH_ERR_ARG;
  if (nparts <= COOP_MAX_PARTS) {
    const int per_sm = ph::occupancy((const void*)k_scan_coop<In, Out>, SCAN_NT, 0);
    const i64 resident = (i64)ph::device_sms() * per_sm;
    if (resident > 0) {
      const int grid = (int)std::min<i64>(nparts, resident);
      void* args[] = {(void*)&in, (void*)&n, (void*)&nparts, (void*)&part, (void*)&out, (void*)&active};
      ph::count_launch();
      if (cudaLaunchCooperativeKernel((const void*)k_scan_coop<In, Out>, grid, SCAN_NT, args, 0, s) != cudaSuccess)
        return PH_ERR_CUDA;
      return PH_OK;
    }
  }
  ph::count_launch();
  ph::launch_pdl(k_scan_reduce<In, Out>, dim3((unsigned)nparts), dim3(SCAN_NT), 0, s, in, n, part, active);
  ph::count_launch();
  ph::launch_pdl(k_scan_partials<Out>, dim3(1), dim3(PART_NT), 0, s, part, nparts, out + n, active);
  ph::count_launch();
  ph::launch_pdl(k_scan_down<In, Out>, dim3((unsigned)nparts), dim3(SCAN_NT), 0, s, in, n, part, out, active);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

// ---------------------------------------------------------------------------
// Radix sort: one-sweep LSD passes with decoupled look-back
// ---------------------------------------------------------------------------
// One kernel histograms all eight digit positions at once; a pass whose
// digit is constant (one bin holds every key) is skipped on the device, and
// the ping-pong parity of every pass follows from the same histogram, so the
// host never synchronises. Each pass is one kernel: a block takes the next
// tile ticket (tickets are handed out in launch order, so every tile a block
// waits on belongs to a block that is already running), ranks its 4096 keys
// stably with warp match-any, publishes its per-digit counts, and sums the
// counts of earlier tiles by looking back until it meets a published
// inclusive prefix. The look-back spin is bounded.
constexpr int RS_NT = 256;
constexpr int RS_WARPS = RS_NT / 32;
// keys per tile: 8 warps x 32 lanes x ROUNDS. Large sorts take 16 rounds
// (4096 keys, few look-back slots); sorts of up to RS_SMALL_MAX keys take 4
// (1024 keys), so that four times as many blocks share the pass and each runs
// a quarter of the serial counting rounds.
constexpr int RS_ROUNDS_LARGE = 16, RS_ROUNDS_SMALL = 4;
constexpr i64 RS_SMALL_MAX = i64(1) << 18;
__host__ __device__ constexpr int rs_tile(int rounds) { return RS_WARPS * 32 * rounds; }
// Lanes of the warp whose digit equals this lane's: one ballot per bit of a
// 9-bit digit (bit 8 marks a lane without a key, so such lanes never match a
// key's digit). Nine ballots issue in fewer cycles than a match-any.
__device__ __forceinline__ u32 warp_peers(u32 d) {
  u32 m = FULL;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const bool bit = (d >> b) & 1u;
    const u32 v = __ballot_sync(FULL, bit);
    m &= bit ? v : ~v;
  }
  return m;
}

constexpr u64 LB_AGG = 1ull << 32, LB_PRE = 2ull << 32;
constexpr int LB_SPIN_LIMIT = 1 << 24;

struct SortCtl {
  u32 ghist[8][256];
  u32 ticket[8];
  int error;
};

__global__ void __launch_bounds__(RS_NT) k_os_hist(const u64* __restrict__ keys, i64 n, int p0, int p1,
                                                  SortCtl* ctl) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ u32 h[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += RS_NT) h[i >> 8][i & 255] = 0;
  __syncthreads();
  // four keys per thread and step, loaded before they are counted
  const i64 step = (i64)gridDim.x * RS_NT * 4;
  for (i64 b = (i64)blockIdx.x * RS_NT * 4 + threadIdx.x; b < n; b += step) {
    u64 k4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) k4[q] = b + q * RS_NT < n ? __ldg(keys + b + q * RS_NT) : 0ull;
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (b + q * RS_NT < n)
        for (int p = p0; p < p1; ++p) atomicAdd(&h[p][(k4[q] >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * 256; i += RS_NT) {
    const u32 v = h[i >> 8][i & 255];
    if (v) atomicAdd(&ctl->ghist[i >> 8][i & 255], v);
  }
}

// Number of active passes before `pass` and whether `pass` itself is active.
__device__ __forceinline__ void pass_plan(const SortCtl* ctl, i64 n, int p0, int pass, int* before,
                                          bool* active, u32* count) {
  // the histogram words first (independent loads), then one barrier per pass
  u32 g[8];
#pragma unroll
  for (int p = 0; p < 8; ++p) g[p] = (p >= p0 && p <= pass) ? ctl->ghist[p][threadIdx.x] : 0u;
  int cnt = 0;
  bool act = false;
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    if (p < p0 || p > pass) continue;
    const int full = __syncthreads_or(g[p] == (u32)n);
    if (p < pass) cnt += !full;
    else act = !full;
  }
  *before = cnt;
  *active = act;
  u32 c = 0;
#pragma unroll
  for (int p = 0; p < 8; ++p)
    if (p == pass) c = g[p];
  *count = c;
}

template <int RS_ROUNDS>
__global__ void __launch_bounds__(RS_NT) k_os_pass(u64* kA, u32* vA, u64* kB, u32* vB, i64 n, int p0,
                                                  int pass, SortCtl* ctl, unsigned long long* lb,
                                                  i64 ntiles) {
  ph::pdl_wait();
  ph::pdl_trigger();
  constexpr int RS_PER_WARP = 32 * RS_ROUNDS;
  constexpr int RS_TILE = rs_tile(RS_ROUNDS);
  __shared__ u32 tile_sh;
  // the first ticket is taken before the plan so that its latency overlaps it
  if (threadIdx.x == 0) tile_sh = atomicAdd(&ctl->ticket[pass], 1u);
  int before;
  bool active;
  u32 v;
  pass_plan(ctl, n, p0, pass, &before, &active, &v);
  if (!active) return;
  const bool srcB = before & 1;
  const u64* ks = srcB ? kB : kA;
  const u32* vs = srcB ? vB : vA;
  u64* kd = srcB ? kA : kB;
  u32* vd = srcB ? vA : vB;
  const int shift = 8 * pass;
  const u64 epoch = (u64)(pass + 1) << 40;
  __shared__ u32 cnt[RS_WARPS][256];
  __shared__ u32 gstart[256];
  __shared__ u32 tbase[256];
  __shared__ u32 wsum[RS_WARPS];
  // exclusive scan of the global digit counts of this pass
  {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u32 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 y = __shfl_up_sync(FULL, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    u32 wp = 0;
    for (int k = 0; k < w; ++k) wp += wsum[k];
    gstart[threadIdx.x] = wp + x - v;
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const u32 lt = lanemask_lt();
  __syncthreads();
  i64 tile = tile_sh;
  for (;;) {
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_NT) cnt[i >> 8][i & 255] = 0;
    __syncthreads();  // every thread has read tile_sh; counters cleared
    if (tile >= ntiles) break;
    // the next ticket is in flight while this tile is sorted; a held ticket
    // never blocks progress, since the lowest unfinished tile is always held
    // by a running block whose earlier tiles are done
    u32 next = 0;
    if (threadIdx.x == 0) next = atomicAdd(&ctl->ticket[pass], 1u);
    const i64 wbase = tile * RS_TILE + (i64)w * RS_PER_WARP;
    u64 key[RS_ROUNDS];
    u32 val[RS_ROUNDS], dig[RS_ROUNDS], pos[RS_ROUNDS];
    // all loads first (independent, in flight together), then the counting rounds
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const i64 i = wbase + r * 32 + lane;
      key[r] = i < n ? __ldg(ks + i) : 0ull;
      val[r] = i < n ? __ldg(vs + i) : 0u;
    }
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const i64 i = wbase + r * 32 + lane;
      const bool ok = i < n;
      const u64 k = key[r];
      const u32 v = val[r];
      const u32 d = ok ? (u32)((k >> shift) & 255u) : 256u;
      const u32 peers = warp_peers(d);
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
    // per-digit tile total; warp counts become exclusive offsets within the tile
    const int dgt = threadIdx.x;
    u32 total = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      const u32 c = cnt[ww][dgt];
      cnt[ww][dgt] = total;
      total += c;
    }
    volatile unsigned long long* slot = lb + tile * 256 + dgt;
    if (tile == 0) {
      *slot = epoch | LB_PRE | total;
      tbase[dgt] = gstart[dgt];
    } else {
      *slot = epoch | LB_AGG | total;
      // look back over the predecessors, eight slots per step (independent
      // loads), summing aggregates until an inclusive prefix is found
      u32 excl = 0;
      i64 t = tile - 1;
      int spins = 0;
      constexpr int LB_BATCH = 8;
      while (t >= 0) {
        unsigned long long cur[LB_BATCH];
#pragma unroll
        for (int q = 0; q < LB_BATCH; ++q)
          cur[q] = (t - q >= 0) ? *(const volatile unsigned long long*)(lb + (t - q) * 256 + dgt) : 0ull;
        bool done = false, wait = false;
        int used = 0;
#pragma unroll
        for (int q = 0; q < LB_BATCH; ++q) {
          if (done || wait || t - q < 0) continue;
          const unsigned long long c = cur[q];
          if ((c & ~((1ull << 40) - 1)) != epoch || ((c >> 32) & 0xffull) == 0) {
            wait = true;  // not published yet: retry from this slot
            continue;
          }
          excl += (u32)(c & 0xffffffffull);
          ++used;
          if (c & LB_PRE) done = true;
        }
        if (done) break;
        t -= used;
        if (wait) {
          if (++spins > LB_SPIN_LIMIT) {
            atomicExch(&ctl->error, 1);
            break;
          }
          __nanosleep(32);
        }
      }
      *slot = epoch | LB_PRE | (excl + total);
      tbase[dgt] = gstart[dgt] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; ++r) {
      const u32 d = dig[r];
      if (d < 256u) {
        const u64 o = (u64)tbase[d] + cnt[w][d] + pos[r];
        kd[o] = key[r];
        vd[o] = val[r];
      }
    }
    if (threadIdx.x == 0) tile_sh = next;
    __syncthreads();
    tile = tile_sh;
  }
}

__global__ void k_os_finish(u64* __restrict__ kA, u32* __restrict__ vA, const u64* __restrict__ kB,
                            const u32* __restrict__ vB, i64 n, int p0, int p1, const SortCtl* ctl) {
  ph::pdl_wait();
  ph::pdl_trigger();
  u32 g[8];
#pragma unroll
  for (int p = 0; p < 8; ++p) g[p] = (p >= p0 && p < p1) ? ctl->ghist[p][threadIdx.x] : 0u;
  int act = 0;
#pragma unroll
  for (int p = 0; p < 8; ++p)
    if (p >= p0 && p < p1) act += !__syncthreads_or(g[p] == (u32)n);
  if (!(act & 1)) return;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    kA[i] = kB[i];
    vA[i] = vB[i];
  }
}

// Cluster form for sorts of up to CS x CS_MAX_CHUNK keys: one cluster of CS
// (16 or 8) blocks holds every (key, value) record in shared memory, block r
// the records at positions [r * chunk, (r + 1) * chunk) of the current order,
// split into one run per warp. A pass counts the digits of each run, reads the
// other blocks' digit counts through distributed shared memory, and writes
// every record straight into the shared memory of the block that holds its
// new position, one 16-byte store per record. Order is stable: block, warp
// run, lane. Two cluster barriers a pass and one launch for the whole sort;
// global memory is touched only by the first load and the last store. A pass
// whose digit is the same for every key is skipped (every block sees the same
// counts, so all skip alike).
constexpr int CS_NT = 512, CS_WARPS = CS_NT / 32;
constexpr i64 CS_MAX_CHUNK = 6144;
constexpr bool CS_PDL = true;  // launched as a dependent of the previous kernel

struct __align__(16) SortRec {
  u64 key;
  u64 val;  // the value in the low 32 bits
};
__device__ __forceinline__ u64 rec_key(const SortRec& r) { return r.key; }
__device__ __forceinline__ u64 rec_key(u64 r) { return r; }

// What a cluster sort reads and writes: (key, value) pairs sorted in place
// (16-byte records), or edges (i, j, dist^2) read from ei/ej/dsq and written
// sorted to oi/oj/od (8-byte records: the packed filtration key
// bits(dist^2) << 32 | j(j-1)/2 + i, from which the edge is rebuilt; exact
// while j(j-1)/2 + i < 2^32, that is for n <= 92682).
struct ClusterSortIO {
  u64* keys;
  u32* vals;
  const i32* ei;
  const i32* ej;
  const float* dsq;
  i32* oi;
  i32* oj;
  float* od;
};

__host__ __device__ constexpr size_t cs_smem_bytes(i64 chunk, size_t rec_bytes) {
  // two record buffers, per-warp digit counts
  return (size_t)chunk * 2 * rec_bytes + (size_t)CS_WARPS * 256 * 4;
}

__device__ __forceinline__ void edge_of_key(u64 key, i32* i, i32* j, float* d) {
  const u64 c = key & 0xffffffffull;
  u64 jj = (u64)((1.0 + sqrt(1.0 + 8.0 * (double)c)) * 0.5);  // j(j-1)/2 <= c < j(j+1)/2
  while (jj > 1 && jj * (jj - 1) / 2 > c) --jj;
  while ((jj + 1) * jj / 2 <= c) ++jj;
  *j = (i32)jj;
  *i = (i32)(c - jj * (jj - 1) / 2);
  *d = __uint_as_float((u32)(key >> 32));
}

template <int CS, bool EDGES>
__global__ void __launch_bounds__(CS_NT, 1) k_cluster_sort(ClusterSortIO io, i64 n, i64 chunk, int p0, int p1) {
  using Rec = typename std::conditional<EDGES, u64, SortRec>::type;
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ __align__(16) unsigned char cs_smem[];
  __shared__ u32 wsum[8];
  __shared__ u32 chist[256];   // this block's digit counts, read by every block
  __shared__ u32 dstart[256];  // where this block's records of each digit go
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  Rec* const rbuf = reinterpret_cast<Rec*>(cs_smem);
  u32* const whist = reinterpret_cast<u32*>(rbuf + 2 * chunk);  // [CS_WARPS][256]
  const i64 lo = (i64)rank * chunk;
  const int cnt = (int)max((i64)0, min(chunk, n - lo));
  const int sub = ((cnt + CS_NT - 1) / CS_NT) * 32;  // records per warp run
  const int wb = min(cnt, w * sub), we = min(cnt, wb + sub);
  u32* const myh = whist + w * 256;
  const u32 lt = lanemask_lt();
  for (int i = tid; i < cnt; i += CS_NT) {
    if constexpr (EDGES) {
      const u64 a = (u64)io.ei[lo + i], b = (u64)io.ej[lo + i];
      rbuf[i] = ((u64)__float_as_uint(io.dsq[lo + i]) << 32) | ((b * (b - 1) / 2 + a) & 0xffffffffull);
    } else {
      rbuf[i] = SortRec{io.keys[lo + i], (u64)io.vals[lo + i]};
    }
  }
  int cur = 0;
  __syncthreads();
  for (int p = p0; p < p1; ++p) {
    const int sh = 8 * p;
    Rec* const R = rbuf + cur * chunk;
    for (int i = lane; i < 256; i += 32) myh[i] = 0;
    __syncwarp();
    for (int b = wb; b < we; b += 32) {
      const int i = b + lane;
      const u32 d = i < we ? (u32)(rec_key(R[i]) >> sh) & 255u : 256u + lane;
      const u32 peers = warp_peers(d);
      if (d < 256u && (peers & lt) == 0) myh[d] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    if (tid < 256) {
      u32 run = 0;
      for (int v = 0; v < CS_WARPS; ++v) {
        const u32 c = whist[v * 256 + tid];
        whist[v * 256 + tid] = run;
        run += c;
      }
      chist[tid] = run;
    }
    cl.sync();  // every block's counts are published
    bool ident = false;
    u32 gs = 0;
    if (tid < 256) {
      // digit d = tid: its count over the cluster and over the blocks before this one
      u32 c[CS];
#pragma unroll
      for (int r = 0; r < CS; ++r) c[r] = *cl.map_shared_rank(chist + tid, r);
      u32 tot = 0, below = 0;
#pragma unroll
      for (int r = 0; r < CS; ++r) {
        tot += c[r];
        if (r < rank) below += c[r];
      }
      ident = tot == (u32)n;
      u32 x = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[w] = x;
      gs = x - tot + below;
    }
    __syncthreads();
    if (tid < 256) {
      for (int v = 0; v < w; ++v) gs += wsum[v];
      dstart[tid] = gs;
    }
    const bool skip = __syncthreads_or(ident);
    if (!skip) {
      Rec* const D = rbuf + (cur ^ 1) * chunk;
      for (int b = wb; b < we; b += 32) {
        const int i = b + lane;
        const bool ok = i < we;
        const Rec r0 = ok ? R[i] : Rec{};
        const u32 d = ok ? (u32)(rec_key(r0) >> sh) & 255u : 256u + lane;
        const u32 peers = warp_peers(d);
        u32 pos = 0;
        if (ok) pos = dstart[d] + myh[d] + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) myh[d] += __popc(peers);
        if (ok && (i64)pos < n) {
          const int r = (int)(pos / (u32)chunk);
          *cl.map_shared_rank(D + (pos - (u32)r * (u32)chunk), r) = r0;
        }
        __syncwarp();
      }
      cur ^= 1;
    }
    cl.sync();  // every record is in place; the counts may be rewritten
  }
  const Rec* const R = rbuf + cur * chunk;
  for (int i = tid; i < cnt; i += CS_NT) {
    if constexpr (EDGES) {
      edge_of_key(R[i], io.oi + lo + i, io.oj + lo + i, io.od + lo + i);
    } else {
      io.keys[lo + i] = R[i].key;
      io.vals[lo + i] = (u32)R[i].val;
    }
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

namespace {
int rs_rounds(i64 n) { return n <= RS_SMALL_MAX ? RS_ROUNDS_SMALL : RS_ROUNDS_LARGE; }

// Blocks in the cluster form's cluster on the current device: 16 where a
// 16-block cluster with full-size buffers can be resident, else 8, 0 when
// neither can. Function attributes belong to a device, so they are set, and
// the answer cached, once per device.
int sort_cluster_size() {
  static std::mutex mu;
  static int cached[64];
  static bool known[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 0;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (known[dev]) return cached[dev];
  known[dev] = true;
  cached[dev] = 0;
  const void* fs[4] = {(const void*)k_cluster_sort<16, false>, (const void*)k_cluster_sort<16, true>,
                       (const void*)k_cluster_sort<8, false>, (const void*)k_cluster_sort<8, true>};
  for (const void* f : fs) {
    if (allow_dynamic_smem(f) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
  }
  cudaFuncSetAttribute(fs[0], cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(fs[1], cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(CS_NT);
    cfg.dynamicSmemBytes = cs_smem_bytes(CS_MAX_CHUNK, sizeof(SortRec));
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, cs == 16 ? fs[0] : fs[2], &cfg) == cudaSuccess && clusters > 0) {
      cached[dev] = cs;
      break;
    }
  }
  cudaGetLastError();
  return cached[dev];
}

// One cluster launch sorting n records by digits [p0, p1); CLUSTER_SORT_NA
// when n is beyond the cluster form (the caller then takes another form).
template <bool EDGES>
int cluster_sort(const ClusterSortIO& io, i64 n, int p0, int p1, cudaStream_t s) {
  const int cs = n <= 16 * CS_MAX_CHUNK ? sort_cluster_size() : 0;
  if (cs == 0 || n > cs * CS_MAX_CHUNK) return CLUSTER_SORT_NA;
  const i64 chunk = (n + cs - 1) / cs;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(CS_NT);
  cfg.dynamicSmemBytes = cs_smem_bytes(chunk, EDGES ? sizeof(u64) : sizeof(SortRec));
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = CS_PDL && dependent_launch_enabled() ? 2 : 1;
  ph::count_launch();
  const cudaError_t e = cs == 16 ? cudaLaunchKernelEx(&cfg, k_cluster_sort<16, EDGES>, io, n, chunk, p0, p1)
                                 : cudaLaunchKernelEx(&cfg, k_cluster_sort<8, EDGES>, io, n, chunk, p0, p1);
  return e == cudaSuccess ? PH_OK : PH_ERR_CUDA;
}
}  // namespace

int cluster_sort_edges(const i32* ei, const i32* ej, const float* dsq, i64 E, i64 n, i32* oi, i32* oj,
                       float* od, cudaStream_t s) {
  if (E < 1 || n > 92682) return CLUSTER_SORT_NA;
  ClusterSortIO io = {};
  io.ei = ei;
  io.ej = ej;
  io.dsq = dsq;
  io.oi = oi;
  io.oj = oj;
  io.od = od;
  return cluster_sort<true>(io, E, 0, 8, s);
}

size_t radix_sort_workspace_bytes(i64 n) {
  const i64 tile = rs_tile(rs_rounds(n));
  const i64 ntiles = (n + tile - 1) / tile + 1;
  return Carve::need((size_t)n * 8) + Carve::need((size_t)n * 4) + Carve::need(sizeof(SortCtl)) +
         Carve::need((size_t)ntiles * 256 * 8);
}

int radix_sort_pairs(u64* keys, u32* vals, i64 n, int begin_bit, int end_bit, void* ws,
                     size_t ws_bytes, cudaStream_t s) {
  if (n < 0 || n >= (i64(1) << 31) || begin_bit < 0 || end_bit > 64 || begin_bit % 8 || end_bit % 8 ||
      begin_bit > end_bit)
    return PH_ERR_ARG;
  if (n <= 1 || begin_bit == end_bit) return PH_OK;
  const int p0 = begin_bit / 8, p1 = end_bit / 8;
  {
    ClusterSortIO io = {};
    io.keys = keys;
    io.vals = vals;
    const int rc = cluster_sort<false>(io, n, p0, p1, s);
    if (rc != CLUSTER_SORT_NA) return rc;
  }
  const int rounds = rs_rounds(n);
  const i64 tile = rs_tile(rounds);
  const i64 ntiles = (n + tile - 1) / tile;
  Carve c(ws, ws_bytes);
  u64* kB = c.take<u64>(n);
  u32* vB = c.take<u32>(n);
  SortCtl* ctl = c.take<SortCtl>(1);
  unsigned long long* lb = c.take<unsigned long long>(ntiles * 256);
  if (!kB || !vB || !ctl || !lb) return PH_ERR_ARG;
  // ctl and lb are adjacent in the workspace: one memset clears both
  const size_t clear = (size_t)((char*)(lb + ntiles * 256) - (char*)ctl);
  ph::zero_async(ctl, clear, s);
  const int gh = (int)std::max<i64>(1, std::min<i64>((n + RS_NT * 4 - 1) / (RS_NT * 4), 592));
  ph::count_launch();
  ph::launch_pdl(k_os_hist, dim3(gh), dim3(RS_NT), 0, s, keys, n, p0, p1, ctl);
  const int gp = (int)std::min<i64>(ntiles, 148 * 4);
  for (int p = p0; p < p1; ++p) {
    ph::count_launch();
    if (rounds == RS_ROUNDS_SMALL)
      ph::launch_pdl(k_os_pass<RS_ROUNDS_SMALL>, dim3(gp), dim3(RS_NT), 0, s, keys, vals, kB, vB, n, p0, p, ctl, lb, ntiles);
    else
      ph::launch_pdl(k_os_pass<RS_ROUNDS_LARGE>, dim3(gp), dim3(RS_NT), 0, s, keys, vals, kB, vB, n, p0, p, ctl, lb, ntiles);
  }
  const int gf = (int)std::max<i64>(1, std::min<i64>((n + 255) / 256, 1184));
  ph::count_launch();
  ph::launch_pdl(k_os_finish, dim3(gf), dim3(256), 0, s, keys, vals, kB, vB, n, p0, p1, ctl);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

}  // namespace ph
