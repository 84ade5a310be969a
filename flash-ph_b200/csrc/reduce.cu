// Z/2 cohomology reduction on the GPU and the persistence rows.
//
// Reference: reduce_h1_gpu.py:159-223 (apparent pairs), cohomology_general.py
// :202-371 (serial residual reduction, Numba on the CPU), reduce_h1_gpu.py
// :574-604 (row assembly).
//
// Columns c = 0..K-1 are processed in the reference's order, descending c;
// the pivot of a column is its smallest row (cofacet rank). The serial
// algorithm adds to a column the stored column that owns its pivot until the
// pivot is unowned. The pivot of every reduced column does not depend on the
// order of additions as long as a column only ever receives columns processed
// before it (larger c): the result is always R = D V with V upper triangular,
// and the pivots of a reduced R are unique. The GPU reducer uses that freedom
// and proceeds in synchronous rounds over all residual columns at once:
//   claim  : each column whose pivot changed does atomicMax(owner[pivot], c)
//   reduce : each column that does not own its pivot adds the owner's column
//            (owners are never written during this phase, so every read is
//            of a stable column) and so strictly raises its pivot
// until a round changes nothing. Then every pivot has exactly one column, so
// the pairs and the essential (emptied) columns are the serial ones, bit for
// bit. Apparent columns own their pivot from the start and never change:
// no column processed before an apparent column can ever contain its pivot.
// Merged columns live in a bump-allocated pool; running out of pool or of the
// round budget sets a status code, no wait is unbounded.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace cg = cooperative_groups;

namespace ph {
namespace {

constexpr int RD_NT = 256;

struct RedCtl {
  int nres;
  int last_change_round;
  int abort;
  int rounds;
  unsigned long long pool_top;
};

// Column content: desc >= 0 -> pool offset; desc < 0 -> cofacet CSR offset -(desc+1).
__device__ __forceinline__ const i32* col_ptr(i64 desc, const i32* cof, const i32* pool) {
  return desc >= 0 ? pool + desc : cof + (-(desc + 1));
}

__global__ void k_classify(const i32* __restrict__ off, const i32* __restrict__ cof, i64 K, i32 col_base,
                           i32 row_base, const uint8_t* __restrict__ skip, const i32* __restrict__ cmf,
                           i32* __restrict__ state, i32* __restrict__ piv, i32* __restrict__ owner,
                           i32* __restrict__ resid, i64* __restrict__ desc, i32* __restrict__ len,
                           uint8_t* __restrict__ changed, RedCtl* ctl) {
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x) {
    const i32 o0 = off[c], o1 = off[c + 1];
    desc[c] = -(i64)o0 - 1;
    len[c] = o1 - o0;
    changed[c] = 1;
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

__device__ __forceinline__ void rd_barrier(cg::grid_group& g) {
  if (gridDim.x == 1) __syncthreads();
  else g.sync();
}

__global__ void __launch_bounds__(RD_NT) k_reduce_rounds(const i32* __restrict__ cof, i32 row_base,
                                                        const i32* __restrict__ resid, i32* __restrict__ piv,
                                                        i32* owner, i64* desc, i32* len, uint8_t* changed,
                                                        i32* pool, i64 pool_cap, RedCtl* ctl, int* status,
                                                        int max_rounds) {
  cg::grid_group g = cg::this_grid();
  const i64 tid = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 nth = (i64)gridDim.x * blockDim.x;
  const i64 nres = ctl->nres;
  if (tid == 0) ctl->last_change_round = -1;
  rd_barrier(g);
  int round = 0;
  for (;; ++round) {
    if (round >= max_rounds) {
      if (tid == 0) set_status(status, PH_ERR_ITER_LIMIT);
      break;
    }
    // claim
    for (i64 r = tid; r < nres; r += nth) {
      const i32 c = resid[r];
      if (changed[c] && len[c] > 0) atomicMax(&owner[piv[c] - row_base], c);
    }
    rd_barrier(g);
    // reduce
    for (i64 r = tid; r < nres; r += nth) {
      const i32 c = resid[r];
      const i32 lc = len[c];
      if (lc == 0) {
        changed[c] = 0;
        continue;
      }
      const i32 o = owner[piv[c] - row_base];
      if (o == c) {
        changed[c] = 0;
        continue;
      }
      if (o < 0) {  // every pivot is claimed before this phase; never taken
        set_status(status, PH_ERR_ARG);
        ctl->abort = 1;
        continue;
      }
      const i32 lo = len[o];
      const i32* A = col_ptr(desc[c], cof, pool);
      const i32* B = col_ptr(desc[o], cof, pool);
      const unsigned long long need = (unsigned long long)lc + (unsigned long long)lo;
      const unsigned long long at = atomicAdd(&ctl->pool_top, need);
      if (at + need > (unsigned long long)pool_cap) {
        set_status(status, PH_ERR_POOL);
        ctl->abort = 1;
        continue;
      }
      i32* out = pool + at;
      int ia = 0, ib = 0, k = 0;
      while (ia < lc && ib < lo) {
        const i32 x = A[ia], y = B[ib];
        if (x < y) {
          out[k++] = x;
          ++ia;
        } else if (y < x) {
          out[k++] = y;
          ++ib;
        } else {
          ++ia;
          ++ib;
        }
      }
      while (ia < lc) out[k++] = A[ia++];
      while (ib < lo) out[k++] = B[ib++];
      desc[c] = (i64)at;
      len[c] = k;
      piv[c] = k ? out[0] : -1;
      changed[c] = 1;
      ctl->last_change_round = round;
    }
    rd_barrier(g);
    if (ctl->abort || ctl->last_change_round != round) break;
  }
  if (tid == 0) ctl->rounds = round + 1;
}

__global__ void k_finish(const i32* __restrict__ resid, const i32* __restrict__ len, i32* __restrict__ state,
                         i32* __restrict__ piv, const RedCtl* ctl, i64* info) {
  const i64 nres = ctl->nres;
  for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < nres; r += (i64)gridDim.x * blockDim.x) {
    const i32 c = resid[r];
    if (len[c] == 0) {
      state[c] = 3;
      piv[c] = -1;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && info) {
    info[0] = ctl->nres;
    info[1] = ctl->rounds;
    info[2] = (i64)ctl->pool_top;
    info[3] = 0;
  }
}

__global__ void k_mark_pivots(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                              uint8_t* __restrict__ flag) {
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x)
    if (state[c] == 1 || state[c] == 2) flag[piv[c] - row_base] = 1;
}

// Row keys: (birth bits, group, order in group); group 0 apparent pairs by
// ascending column, 1 reduced pairs and 2 essential columns by descending
// column; columns without a row get the largest key.
__global__ void k_row_keys(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                           const float* __restrict__ filt, const i32* __restrict__ col_m,
                           const i32* __restrict__ row_m, u64* __restrict__ keys, u32* __restrict__ vals,
                           unsigned long long* nrows) {
  unsigned long long cnt = 0;
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x) {
    const i32 st = state[c];
    u64 key = ~0ull;
    if (st != 0) {
      const float fb = filt[col_m ? col_m[c] : (i32)c];
      bool keep = true;
      u64 group = 2;
      if (st == 1 || st == 2) {
        const float fd = filt[row_m[piv[c] - row_base]];
        keep = fd > fb;
        group = (st == 1) ? 0 : 1;
      }
      if (keep) {
        const u64 ord = group == 0 ? (u64)c : (u64)(K - 1 - c);
        key = ((u64)float_bits(fb) << 32) | (group << 30) | ord;
        ++cnt;
      }
    }
    keys[c] = key;
    vals[c] = (u32)c;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nrows, cnt);
}

__global__ void k_rows_out(const u32* __restrict__ vals, const i32* __restrict__ state,
                           const i32* __restrict__ piv, i32 row_base, const float* __restrict__ filt,
                           const i32* __restrict__ col_m, const i32* __restrict__ row_m,
                           const unsigned long long* nrows, float* __restrict__ rows, i64* d_nrows) {
  const i64 n = (i64)*nrows;
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (i64)gridDim.x * blockDim.x) {
    const i32 c = (i32)vals[p];
    rows[2 * p] = filt[col_m ? col_m[c] : c];
    rows[2 * p + 1] = state[c] == 3 ? __int_as_float(0x7f800000) : filt[row_m[piv[c] - row_base]];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_nrows = n;
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" size_t ph_reduce_workspace_bytes(int64_t K, int64_t R) {
  return Carve::need((size_t)R * 4) + Carve::need((size_t)K * 4) + Carve::need((size_t)K * 8) +
         Carve::need((size_t)K * 4) + Carve::need((size_t)K) + Carve::need(sizeof(RedCtl));
}

extern "C" int ph_reduce(const int32_t* cof_off, const int32_t* cof_data, int64_t K, int32_t col_base,
                         int64_t R, int32_t row_base, const uint8_t* skip, const int32_t* row_cmf,
                         int32_t* col_state, int32_t* col_piv, int32_t* pool, int64_t pool_cap,
                         int64_t* d_info, int* d_status, void* workspace, size_t workspace_bytes,
                         void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0 || R < 0 || pool_cap < 0) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 31) || R >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  if (K == 0) {
    if (d_info) cudaMemsetAsync(d_info, 0, 4 * sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  i32* owner = c.take<i32>(std::max<i64>(R, 1));
  i32* resid = c.take<i32>(K);
  i64* desc = c.take<i64>(K);
  i32* len = c.take<i32>(K);
  uint8_t* changed = c.take<uint8_t>(K);
  RedCtl* ctl = c.take<RedCtl>(1);
  if (!owner || !resid || !desc || !len || !changed || !ctl) return PH_ERR_ARG;
  cudaMemsetAsync(owner, 0xff, sizeof(i32) * std::max<i64>(R, 1), s);
  cudaMemsetAsync(ctl, 0, sizeof(RedCtl), s);
  ph::count_launch();
  k_classify<<<grid_for(K), 256, 0, s>>>(cof_off, cof_data, K, col_base, row_base, skip, row_cmf, col_state,
                                         col_piv, owner, resid, desc, len, changed, ctl);
  PH_CHECK_LAUNCH();
  int max_rounds = 1 << 22;
  // The residual count is only known on the device; size the grid for K.
  if (K <= 4 * RD_NT) {
    ph::count_launch();
    k_reduce_rounds<<<1, RD_NT, 0, s>>>(cof_data, row_base, resid, col_piv, owner, desc, len, changed, pool,
                                        pool_cap, ctl, d_status, max_rounds);
  } else {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_reduce_rounds, RD_NT, 0);
    if (per_sm < 1) return PH_ERR_CUDA;
    const int blocks = (int)std::max<i64>(2, std::min<i64>((K + RD_NT * 4 - 1) / (RD_NT * 4), (i64)sms * per_sm));
    const i32* cof = cof_data;
    void* args[] = {(void*)&cof,     (void*)&row_base, (void*)&resid,  (void*)&col_piv, (void*)&owner,
                    (void*)&desc,    (void*)&len,      (void*)&changed, (void*)&pool,   (void*)&pool_cap,
                    (void*)&ctl,     (void*)&d_status, (void*)&max_rounds};
    ph::count_launch();
    if (cudaLaunchCooperativeKernel((const void*)k_reduce_rounds, blocks, RD_NT, args, 0, s) != cudaSuccess)
      return PH_ERR_CUDA;
  }
  ph::count_launch();
  k_finish<<<grid_for(K), 256, 0, s>>>(resid, len, col_state, col_piv, ctl, d_info);
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

extern "C" size_t ph_persistence_rows_workspace_bytes(int64_t K) {
  return Carve::need((size_t)K * 8) + Carve::need((size_t)K * 4) + Carve::need(8) + radix_sort_workspace_bytes(K);
}

extern "C" int ph_persistence_rows(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                                   const float* filt, const int32_t* col_m, const int32_t* row_m, float* out_rows,
                                   int64_t* d_nrows, void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 30)) return PH_ERR_OVERFLOW;
  if (K == 0) {
    cudaMemsetAsync(d_nrows, 0, sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(K);
  u32* vals = c.take<u32>(K);
  unsigned long long* cnt = c.take<unsigned long long>(1);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(K));
  if (!keys || !vals || !cnt || !rws) return PH_ERR_ARG;
  cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
  ph::count_launch();
  k_row_keys<<<grid_for(K), 256, 0, s>>>(col_state, col_piv, K, row_base, filt, col_m, row_m, keys, vals, cnt);
  PH_TRY(radix_sort_pairs(keys, vals, K, 0, 64, rws, radix_sort_workspace_bytes(K), s));
  ph::count_launch();
  k_rows_out<<<grid_for(K), 256, 0, s>>>(vals, col_state, col_piv, row_base, filt, col_m, row_m, cnt, out_rows,
                                         d_nrows);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
