// H0: minimum spanning forest (reference: boruvka.py:17-113) and the H0 rows
// (persistence.py:169-192).
//
// One cooperative kernel runs all Boruvka rounds with grid-wide barriers
// instead of one host round trip per round. Weights are the edge ranks, which
// are distinct, so the forest is unique and equals the reference's. Each
// round: every root takes the lowest-ranked edge leaving it (atomicMin over
// the edges), roots hook along their choice (of a mutual pair only the larger
// root hooks, so no cycle can form), and parents are flattened with
// concurrent path halving. Every loop is bounded; overruns set
// PH_ERR_ITER_LIMIT in the device status word instead of spinning.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace cg = cooperative_groups;

namespace ph {
namespace {

constexpr int MST_NT = 512;

struct MstCtl {
  int last_hook_round;
  int abort;
  long long ncomp;
};

__device__ __forceinline__ void barrier(cg::grid_group& g) {
  if (gridDim.x == 1) __syncthreads();
  else g.sync();
}

__device__ __forceinline__ i32 find_root(i32* parent, i32 v, int* status, MstCtl* ctl) {
  // path halving; concurrent writers only ever store an ancestor
  for (int it = 0; it < (1 << 26); ++it) {
    const i32 p = parent[v];
    const i32 gp = parent[p];
    if (p == gp) return p;
    parent[v] = gp;
    v = gp;
  }
  set_status(status, PH_ERR_ITER_LIMIT);
  ctl->abort = 1;
  return v;
}

__global__ void __launch_bounds__(MST_NT) k_mst(const i32* __restrict__ ei, const i32* __restrict__ ej,
                                               i64 E, i64 n, i32* parent, i32* best, i32* other,
                                               i32* minv, uint8_t* mst, i32* comp, MstCtl* ctl,
                                               int* status, int max_rounds) {
  cg::grid_group g = cg::this_grid();
  const i64 tid = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 nth = (i64)gridDim.x * blockDim.x;
  for (i64 v = tid; v < n; v += nth) {
    parent[v] = (i32)v;
    minv[v] = INT_MAX;
  }
  for (i64 e = tid; e < E; e += nth) mst[e] = 0;
  if (tid == 0) {
    ctl->last_hook_round = -1;
    ctl->abort = 0;
    ctl->ncomp = 0;
  }
  barrier(g);
  for (int round = 0;; ++round) {
    if (round >= max_rounds) {
      if (tid == 0) set_status(status, PH_ERR_ITER_LIMIT);
      break;
    }
    for (i64 v = tid; v < n; v += nth) best[v] = INT_MAX;
    barrier(g);
    // lowest-ranked edge leaving each root (parents are flat here)
    for (i64 e = tid; e < E; e += nth) {
      const i32 ru = parent[ei[e]], rv = parent[ej[e]];
      if (ru != rv) {
        atomicMin(&best[ru], (i32)e);
        atomicMin(&best[rv], (i32)e);
      }
    }
    barrier(g);
    for (i64 r = tid; r < n; r += nth) {
      const i32 e = best[r];
      if (e != INT_MAX && parent[r] == r) {
        const i32 a = parent[ei[e]], b = parent[ej[e]];
        other[r] = (a == (i32)r) ? b : a;
      }
    }
    barrier(g);
    for (i64 r = tid; r < n; r += nth) {
      const i32 e = best[r];
      if (e == INT_MAX || parent[r] != r) continue;
      const i32 o = other[r];
      mst[e] = 1;
      if (best[o] == e && o > (i32)r) continue;  // mutual choice: the larger root hooks
      parent[r] = o;
      ctl->last_hook_round = round;
    }
    barrier(g);
    // roots are never written while flattening, so each vertex ends on its root
    for (i64 v = tid; v < n; v += nth) parent[v] = find_root(parent, (i32)v, status, ctl);
    barrier(g);
    if (ctl->abort || ctl->last_hook_round != round) break;
  }
  // labels: smallest vertex of each component, and the component count
  long long roots = 0;
  for (i64 v = tid; v < n; v += nth) {
    atomicMin(&minv[parent[v]], (i32)v);
    roots += (parent[v] == (i32)v);
  }
  for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(0xffffffffu, roots, o);
  if ((threadIdx.x & 31) == 0 && roots) atomicAdd((unsigned long long*)&ctl->ncomp, (unsigned long long)roots);
  barrier(g);
  for (i64 v = tid; v < n; v += nth) comp[v] = minv[parent[v]];
}

__global__ void k_copy_ncomp(const MstCtl* ctl, int64_t* out) { *out = ctl->ncomp; }

__global__ void k_h0_rows(const float* __restrict__ filt, const uint8_t* __restrict__ mst,
                          const i32* __restrict__ pos, i64 E, i64 n, float* __restrict__ rows) {
  const i64 cnt = pos[E];
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x)
    if (mst[e]) {
      rows[2 * pos[e]] = 0.0f;
      rows[2 * pos[e] + 1] = filt[e];
    }
  for (i64 r = cnt + (i64)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (i64)gridDim.x * blockDim.x) {
    rows[2 * r] = 0.0f;
    rows[2 * r + 1] = __int_as_float(0x7f800000);
  }
}

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" size_t ph_boruvka_workspace_bytes(int64_t n, int64_t E) {
  (void)E;
  return 4 * Carve::need((size_t)n * 4) + Carve::need(sizeof(MstCtl));
}

extern "C" int ph_boruvka_mst(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                              uint8_t* mst_mask, int32_t* comp, int64_t* d_ncomp, int* d_status,
                              void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || E < 0 || n >= (int64_t(1) << 31) || E >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  if (n == 0) {
    cudaMemsetAsync(d_ncomp, 0, sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  i32* parent = c.take<i32>(n);
  i32* best = c.take<i32>(n);
  i32* other = c.take<i32>(n);
  i32* minv = c.take<i32>(n);
  MstCtl* ctl = c.take<MstCtl>(1);
  if (!parent || !best || !other || !minv || !ctl) return PH_ERR_ARG;
  const i64 work = std::max<i64>(n, E);
  int max_rounds = 2;
  while ((i64(1) << (max_rounds - 2)) < n && max_rounds < 64) ++max_rounds;
  max_rounds += 4;
  if (work <= 4 * MST_NT * 8) {
    ph::count_launch();
    k_mst<<<1, MST_NT, 0, s>>>(edge_i, edge_j, E, n, parent, best, other, minv, mst_mask, comp, ctl,
                               d_status, max_rounds);
  } else {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mst, MST_NT, 0);
    if (per_sm < 1) return PH_ERR_CUDA;
    const i64 want = (work + MST_NT * 4 - 1) / (MST_NT * 4);
    const int blocks = (int)std::max<i64>(2, std::min<i64>(want, (i64)sms * per_sm));
    void* args[] = {(void*)&edge_i, (void*)&edge_j, (void*)&E,      (void*)&n,      (void*)&parent,
                    (void*)&best,   (void*)&other,  (void*)&minv,   (void*)&mst_mask, (void*)&comp,
                    (void*)&ctl,    (void*)&d_status, (void*)&max_rounds};
    ph::count_launch();
    if (cudaLaunchCooperativeKernel((const void*)k_mst, blocks, MST_NT, args, 0, s) != cudaSuccess)
      return PH_ERR_CUDA;
  }
  ph::count_launch();
  k_copy_ncomp<<<1, 1, 0, s>>>(ctl, d_ncomp);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_h0_rows_workspace_bytes(int64_t E) {
  return Carve::need((size_t)(E + 1) * 4) + scan_workspace_bytes(E);
}

extern "C" int ph_h0_rows(const float* edge_filt, const uint8_t* mst_mask, int64_t E, int64_t n,
                          float* out_rows, void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || n < 0) return PH_ERR_ARG;
  if (n == 0) return PH_OK;
  Carve c(workspace, workspace_bytes);
  i32* pos = c.take<i32>(E + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(E));
  if (!pos || !sws) return PH_ERR_ARG;
  PH_TRY(scan_exclusive_u8_i32(mst_mask, pos, E, sws, scan_workspace_bytes(E), s));
  const i64 work = std::max<i64>(E, n);
  const int g = (int)std::max<i64>(1, std::min<i64>((work + 255) / 256, 148 * 8));
  ph::count_launch();
  k_h0_rows<<<g, 256, 0, s>>>(edge_filt, mst_mask, pos, E, n, out_rows);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
