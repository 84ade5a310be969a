// Z/2 cohomology reduction on the GPU and the persistence rows.
//
// Reference: reduce_h1_gpu.py:159-223 (apparent pairs), cohomology_general.py
// :202-371 (serial residual reduction, Numba on the CPU), reduce_h1_gpu.py
// :574-604 (row assembly).
//
// Columns c = 0..K-1 are processed in the reference's order, descending c;
// the pivot of a column is its smallest row (cofacet rank). The serial
// algorithm adds to a column the stored column that owns its pivot until the
// pivot is unowned. The pivots of the reduced matrix do not depend on the
// order of additions as long as a column only ever receives columns processed
// before it (larger c): the result is always R = D V with V upper triangular,
// and the pivots (hence the pairs and the set of emptied columns) of any such
// reduced R are unique. The GPU reducer uses that freedom and runs lock-free:
// each warp takes a residual column, keeps it in shared memory and adds the
// column that owns its current pivot while that owner is a larger column.
// When the pivot is free or held by a smaller column, the warp publishes the
// column (immutable pool copy, then its descriptor, then a fence) and claims
// the pivot with atomicMax. A smaller column it displaces is taken over by the
// same warp and reduced further. No warp ever waits for another; every loop
// is bounded; running out of pool sets a status code. Apparent columns own
// their pivot from the start and are never displaced (no column processed
// before an apparent column can contain its pivot).
#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace ph {
namespace {

// Few warps with large shared buffers: the reduction is bound by the latency
// of its dependency chains, not by parallel width, and a working column that
// outgrows its shared buffer falls back to global memory (slow binary
// searches), so the buffers are sized to hold long columns.
constexpr int RD_NT = 128;
constexpr int RD_WARPS = RD_NT / 32;
constexpr int RD_CAP = 4096;  // per-warp shared buffers (entries): two working copies + the added column
constexpr size_t RD_SMEM = (size_t)RD_WARPS * 3 * RD_CAP * sizeof(int32_t);
constexpr unsigned FULL = 0xffffffffu;
constexpr u64 D_CSR = 1ull << 63;
constexpr u64 D_OFF = (1ull << 40) - 1;
constexpr int D_LEN_MAX = (1 << 23) - 1;

struct RedCtl {
  int nres;
  int next;
  int abort;
  int pad;
  unsigned long long pool_top;
  unsigned long long merges;
  unsigned long long takeovers;
};

// Column descriptor: bit 63 = content in the cofacet CSR (else in the pool),
// bits 40..62 = length, bits 0..39 = offset.
__device__ __forceinline__ u64 pack_desc(bool csr, u64 len, u64 off) {
  return (csr ? D_CSR : 0ull) | (len << 40) | off;
}
__device__ __forceinline__ int dlen(u64 d) { return (int)((d >> 40) & (u64)D_LEN_MAX); }
__device__ __forceinline__ const i32* dptr(u64 d, const i32* cof, const i32* pool) {
  return ((d & D_CSR) ? cof : pool) + (d & D_OFF);
}

__global__ void k_classify(const i32* __restrict__ off, const i32* __restrict__ cof, i64 K, i32 col_base,
                           i32 row_base, const uint8_t* __restrict__ skip, const i32* __restrict__ cmf,
                           i32* __restrict__ state, i32* __restrict__ piv, i32* __restrict__ owner,
                           i32* __restrict__ resid, u64* __restrict__ desc, RedCtl* ctl, int* status) {
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x) {
    const i32 o0 = off[c], o1 = off[c + 1];
    if (o1 - o0 > D_LEN_MAX) set_status(status, PH_ERR_OVERFLOW);
    desc[c] = pack_desc(true, (u64)(o1 - o0), (u64)o0);
    if (skip && skip[c]) {
      state[c] = 0;
      piv[c] = -1;
    } else if (o0 == o1) {
      state[c] = 3;
      piv[c] = -1;
    } else {
      const i32 t = cof[o0];
      piv[c] = t;
      if (cmf[t - row_base] == col_base + (i32)c) {
        state[c] = 1;
        owner[t - row_base] = (i32)c;
      } else {
        state[c] = 2;
        resid[atomicAdd(&ctl->nres, 1)] = (i32)c;
      }
    }
  }
}

// Loads that must see data written by other SMs during this kernel go to L2.
template <bool G>
__device__ __forceinline__ i32 ld(const i32* p) {
  if (G) return __ldcg(p);
  return *p;
}

template <bool G>
__device__ __forceinline__ int lower_bound_t(const i32* a, int n, i32 x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld<G>(a + mid) < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// out = A xor B for sorted lists of distinct ranks, computed by the whole
// warp: every element looks itself up in the other list; a surviving a_i
// goes to position i + lower_bound_B(a_i) - 2 * #(a_k in B, k < i), and
// symmetrically for B. Returns the (warp-uniform) output length.
template <bool AG, bool BG>
__device__ int warp_symdiff(const i32* A, int na, const i32* B, int nb, i32* out) {
  const int lane = threadIdx.x & 31;
  const u32 lt = lanemask_lt();
  int common = 0;
  for (int base = 0; base < na; base += 32) {
    const int i = base + lane;
    bool in = false;
    int lb = 0;
    i32 x = 0;
    if (i < na) {
      x = ld<AG>(A + i);
      lb = lower_bound_t<BG>(B, nb, x);
      in = lb < nb && ld<BG>(B + lb) == x;
    }
    const u32 m = __ballot_sync(FULL, in);
    const int ci = common + __popc(m & lt);
    if (i < na && !in) out[i + lb - 2 * ci] = x;
    common += __popc(m);
  }
  int cb = 0;
  for (int base = 0; base < nb; base += 32) {
    const int j = base + lane;
    bool in = false;
    int la = 0;
    i32 y = 0;
    if (j < nb) {
      y = ld<BG>(B + j);
      la = lower_bound_t<AG>(A, na, y);
      in = la < na && ld<AG>(A + la) == y;
    }
    const u32 m = __ballot_sync(FULL, in);
    const int dj = cb + __popc(m & lt);
    if (j < nb && !in) out[j + la - 2 * dj] = y;
    cb += __popc(m);
  }
  return na + nb - 2 * common;
}

__device__ __forceinline__ int symdiff(const i32* A, bool ag, int na, const i32* B, bool bg, int nb, i32* out) {
  if (ag) return bg ? warp_symdiff<true, true>(A, na, B, nb, out) : warp_symdiff<true, false>(A, na, B, nb, out);
  return bg ? warp_symdiff<false, true>(A, na, B, nb, out) : warp_symdiff<false, false>(A, na, B, nb, out);
}

// Bump allocation in the pool (lane 0), broadcast to the warp; ~0 on overflow.
__device__ __forceinline__ unsigned long long pool_alloc(RedCtl* ctl, i64 cap, int n, int* status) {
  unsigned long long at = 0;
  if ((threadIdx.x & 31) == 0) {
    at = atomicAdd(&ctl->pool_top, (unsigned long long)n);
    if (at + (unsigned long long)n > (unsigned long long)cap) {
      set_status(status, PH_ERR_POOL);
      atomicExch(&ctl->abort, 1);
      at = ~0ull;
    }
  }
  return __shfl_sync(FULL, at, 0);
}

__global__ void __launch_bounds__(RD_NT) k_reduce(const i32* __restrict__ cof, i32 row_base,
                                                 const i32* __restrict__ resid, u64* desc, i32* owner, i32* pool,
                                                 i64 pool_cap, RedCtl* ctl, int* status, int max_steps) {
  extern __shared__ i32 rd_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  i32* sWw[2] = {rd_smem + (size_t)w * 3 * RD_CAP, rd_smem + (size_t)w * 3 * RD_CAP + RD_CAP};
  i32* sBw = rd_smem + (size_t)w * 3 * RD_CAP + 2 * RD_CAP;
  const int nres = ctl->nres;
  volatile u64* vdesc = desc;
  volatile i32* vowner = owner;
  volatile int* vabort = &ctl->abort;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(&ctl->next, 1);
    idx = __shfl_sync(FULL, idx, 0);
    if (idx >= nres || *vabort) break;
    i32 c = resid[idx];
    u64 dc = vdesc[c];
    // working column: shared buffer sWw[cur] or, when too long, global
    int cur = 0;
    int k = dlen(dc);
    const i32* W;
    bool wg;          // W is in global memory
    bool published;   // dc describes W exactly (nothing to write before a claim)
    auto load_work = [&](u64 d) {
      k = dlen(d);
      const i32* src = dptr(d, cof, pool);
      if (k <= RD_CAP) {
        for (int i = lane; i < k; i += 32) sWw[cur][i] = __ldcg(src + i);
        __syncwarp();
        W = sWw[cur];
        wg = false;
      } else {
        W = src;
        wg = true;
      }
      dc = d;
      published = true;
    };
    load_work(dc);
    for (int step = 0;; ++step) {
      if (step >= max_steps) {
        if (lane == 0) set_status(status, PH_ERR_ITER_LIMIT);
        atomicExch(&ctl->abort, 1);
        break;
      }
      if (k == 0) {
        if (lane == 0) vdesc[c] = pack_desc(false, 0, 0);
        break;
      }
      const i32 p = wg ? __ldcg(W) : W[0];
      i32 o = vowner[p - row_base];
      if (o < c) {
        // publish W, then claim p
        if (!published) {
          const unsigned long long at = pool_alloc(ctl, pool_cap, k, status);
          if (at == ~0ull) break;
          for (int i = lane; i < k; i += 32) pool[at + i] = wg ? __ldcg(W + i) : W[i];
          dc = pack_desc(false, (u64)k, at);
          published = true;
        }
        __threadfence();
        __syncwarp();
        i32 old = 0;
        if (lane == 0) {
          vdesc[c] = dc;
          __threadfence();
          old = atomicMax(&owner[p - row_base], c);
        }
        old = __shfl_sync(FULL, old, 0);
        if (old < c) {
          if (old < 0) break;  // claimed a free pivot: this work item is done
          // displaced a smaller column: take it over
          if (lane == 0) atomicAdd(&ctl->takeovers, 1ull);
          c = old;
          __threadfence();
          load_work(vdesc[c]);
          continue;
        }
        o = old;  // a larger column got there first
      }
      if (o == c) {  // cannot happen: a column never owns a pivot it is still reducing
        if (lane == 0) set_status(status, PH_ERR_ARG);
        break;
      }
      // add the larger owner o
      __threadfence();
      const u64 od = vdesc[o];
      const int lb = dlen(od);
      const i32* Bsrc = dptr(od, cof, pool);
      const i32* B;
      bool bg;
      if (lb <= RD_CAP) {
        for (int i = lane; i < lb; i += 32) sBw[i] = __ldcg(Bsrc + i);
        __syncwarp();
        B = sBw;
        bg = false;
      } else {
        B = Bsrc;
        bg = true;
      }
      i32* out;
      bool og;
      unsigned long long at = 0;
      if (k + lb <= RD_CAP) {
        out = sWw[cur ^ 1];
        og = false;
      } else {
        at = pool_alloc(ctl, pool_cap, k + lb, status);
        if (at == ~0ull) break;
        out = pool + at;
        og = true;
      }
      const int m = symdiff(W, wg, k, B, bg, lb, out);
      __syncwarp();
      if (lane == 0) atomicAdd(&ctl->merges, 1ull);
      k = m;
      if (og) {
        __threadfence();
        W = out;
        wg = true;
        dc = pack_desc(false, (u64)k, at);
        published = true;
      } else {
        cur ^= 1;
        W = sWw[cur];
        wg = false;
        published = false;
      }
    }
  }
}

__global__ void k_finish(const i32* __restrict__ cof, const i32* __restrict__ pool, const i32* __restrict__ resid,
                         const u64* __restrict__ desc, i32* __restrict__ state, i32* __restrict__ piv,
                         const RedCtl* ctl, i64* info) {
  const i64 nres = ctl->nres;
  for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < nres; r += (i64)gridDim.x * blockDim.x) {
    const i32 c = resid[r];
    const u64 d = desc[c];
    if (dlen(d) == 0) {
      state[c] = 3;
      piv[c] = -1;
    } else {
      state[c] = 2;
      piv[c] = dptr(d, cof, pool)[0];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && info) {
    info[0] = ctl->nres;
    info[1] = (i64)ctl->merges;
    info[2] = (i64)ctl->pool_top;
    info[3] = (i64)ctl->takeovers;
  }
}

__global__ void k_mark_pivots(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                              uint8_t* __restrict__ flag) {
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x)
    if (state[c] == 1 || state[c] == 2) flag[piv[c] - row_base] = 1;
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" size_t ph_reduce_workspace_bytes(int64_t K, int64_t R) {
  return Carve::need((size_t)R * 4) + Carve::need((size_t)K * 4) + Carve::need((size_t)K * 8) +
         Carve::need(sizeof(RedCtl));
}

extern "C" int ph_reduce(const int32_t* cof_off, const int32_t* cof_data, int64_t K, int32_t col_base,
                         int64_t R, int32_t row_base, const uint8_t* skip, const int32_t* row_cmf,
                         int32_t* col_state, int32_t* col_piv, int32_t* pool, int64_t pool_cap,
                         int64_t* d_info, int* d_status, void* workspace, size_t workspace_bytes,
                         void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0 || R < 0 || pool_cap < 0) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 31) || R >= (int64_t(1) << 31) || pool_cap >= (int64_t(1) << 40))
    return PH_ERR_OVERFLOW;
  if (K == 0) {
    if (d_info) cudaMemsetAsync(d_info, 0, 4 * sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  i32* owner = c.take<i32>(std::max<i64>(R, 1));
  i32* resid = c.take<i32>(K);
  u64* desc = c.take<u64>(K);
  RedCtl* ctl = c.take<RedCtl>(1);
  if (!owner || !resid || !desc || !ctl) return PH_ERR_ARG;
  cudaMemsetAsync(owner, 0xff, sizeof(i32) * std::max<i64>(R, 1), s);
  cudaMemsetAsync(ctl, 0, sizeof(RedCtl), s);
  ph::count_launch();
  k_classify<<<grid_for(K), 256, 0, s>>>(cof_off, cof_data, K, col_base, row_base, skip, row_cmf, col_state,
                                         col_piv, owner, resid, desc, ctl, d_status);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(k_reduce, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RD_SMEM) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  int occ = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_reduce, RD_NT, RD_SMEM);
  // residual count is known only on the device; K bounds it. Blocks are
  // persistent (a shared work counter), so only resident blocks are launched.
  const int blocks = (int)std::max<i64>(1, std::min<i64>((K + RD_WARPS - 1) / RD_WARPS, (i64)sms * std::max(occ, 1)));
  ph::count_launch();
  k_reduce<<<blocks, RD_NT, RD_SMEM, s>>>(cof_data, row_base, resid, desc, owner, pool, pool_cap, ctl, d_status,
                                    1 << 24);
  ph::count_launch();
  k_finish<<<grid_for(K), 256, 0, s>>>(cof_data, pool, resid, desc, col_state, col_piv, ctl, d_info);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_mark_pivots(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                              uint8_t* row_flag, int64_t R, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0 || R < 0) return PH_ERR_ARG;
  if (R > 0) cudaMemsetAsync(row_flag, 0, (size_t)R, s);
  if (K > 0) {
    ph::count_launch();
    k_mark_pivots<<<grid_for(K), 256, 0, s>>>(col_state, col_piv, K, row_base, row_flag);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_persistence_rows_workspace_bytes(int64_t K) { return rows_nosort_workspace_bytes(K); }

extern "C" int ph_persistence_rows(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                                   const float* filt, const int32_t* col_m, const int32_t* row_m, float* out_rows,
                                   int64_t* d_nrows, void* workspace, size_t workspace_bytes, void* stream) {
  if (K < 0) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  return rows_nosort(col_state, col_piv, K, row_base, filt, col_m, row_m, nullptr, 1, out_rows, nullptr, d_nrows,
                     workspace, workspace_bytes, (cudaStream_t)stream);
}
