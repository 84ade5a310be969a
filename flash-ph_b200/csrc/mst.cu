// H0: minimum spanning forest (reference: boruvka.py:17-113) and the H0 rows
// (persistence.py:169-192).
//
// One cooperative kernel runs all Boruvka rounds with grid-wide barriers
// instead of one host round trip per round, two barriers a round. Weights are
// the edge ranks, which are distinct, so the forest is unique and equals the
// reference's. Each round: every edge between two components offers itself to
// both roots (atomicMin of its rank); after the barrier every root that
// received an offer marks that edge and merges the two components with a
// lock-free union (CAS on the larger root, which is linked under the smaller).
// The chosen edges all belong to the unique forest, so they never close a
// cycle; a mutual choice is one edge, merged once. Parents only ever point to
// a smaller vertex, so finds (path halving) terminate and a component's root
// is its smallest vertex, which is the reference's component label. Every loop
// is bounded; overruns set PH_ERR_ITER_LIMIT in the device status word
// instead of spinning.
#include <cooperative_groups.h>

#include <mutex>

#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace cg = cooperative_groups;

namespace ph {
namespace {

constexpr int MST_NT = 512;
// forest mask value of an edge found inside one component: skipped by every
// later round (components only merge), reset to 0 before the kernel ends
constexpr uint8_t MST_DROPPED = 2;

struct MstCtl {
  int last_offer_round;
  int abort;
  long long ncomp;
};

__device__ __forceinline__ void barrier(cg::grid_group& g) {
  if (gridDim.x == 1) __syncthreads();
  else g.sync();
}

// root of v by path halving; parent[] is read past the L1 (other blocks link
// roots concurrently) and only ever rewritten to an ancestor
__device__ __forceinline__ i32 find_root(i32* parent, i32 v, int* status, MstCtl* ctl) {
  volatile i32* par = parent;
  for (int it = 0; it < (1 << 26); ++it) {
    const i32 p = par[v];
    if (p == v) return v;
    const i32 gp = par[p];
    if (gp == p) return p;
    par[v] = gp;
    v = gp;
  }
  set_status(status, PH_ERR_ITER_LIMIT);
  ctl->abort = 1;
  return v;
}

__global__ void __launch_bounds__(MST_NT) k_mst(const i32* __restrict__ ei, const i32* __restrict__ ej,
                                               i64 E, i64 n, i32* parent, i32* best, uint8_t* mst,
                                               i32* comp, MstCtl* ctl, int* status, int max_rounds) {
  ph::pdl_wait();
  ph::pdl_trigger();
  cg::grid_group g = cg::this_grid();
  const i64 tid = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 nth = (i64)gridDim.x * blockDim.x;
  for (i64 v = tid; v < n; v += nth) {
    parent[v] = (i32)v;
    best[v] = INT_MAX;
  }
  for (i64 e = tid; e < E; e += nth) mst[e] = 0;
  if (tid == 0) {
    ctl->last_offer_round = -1;
    ctl->abort = 0;
    ctl->ncomp = 0;
  }
  barrier(g);
  for (int round = 0;; ++round) {
    if (round >= max_rounds) {
      if (tid == 0) set_status(status, PH_ERR_ITER_LIMIT);
      break;
    }
    // offers: the lowest-ranked edge leaving each root (no links in this phase)
    bool offered = false;
    for (i64 e = tid; e < E; e += nth) {
      const uint8_t st = mst[e];
      if (st == MST_DROPPED) continue;
      const i32 ru = find_root(parent, ei[e], status, ctl), rv = find_root(parent, ej[e], status, ctl);
      if (ru != rv) {
        if ((i32)e < *(volatile i32*)&best[ru]) atomicMin(&best[ru], (i32)e);
        if ((i32)e < *(volatile i32*)&best[rv]) atomicMin(&best[rv], (i32)e);
        offered = true;
      } else if (st == 0) {
        mst[e] = MST_DROPPED;  // inside one component for good: later rounds skip it
      }
    }
    if (__syncthreads_or(offered) && threadIdx.x == 0) ctl->last_offer_round = round;
    barrier(g);
    if (*(volatile int*)&ctl->abort || *(volatile int*)&ctl->last_offer_round != round) break;
    // links: each root with an offer marks it and merges the two components
    for (i64 v = tid; v < n; v += nth) {
      const i32 e = best[v];
      if (e == INT_MAX) continue;
      best[v] = INT_MAX;
      mst[e] = 1;
      i32 a = ei[e], b = ej[e];
      for (int it = 0;; ++it) {
        if (it >= (1 << 20)) {
          set_status(status, PH_ERR_ITER_LIMIT);
          ctl->abort = 1;
          break;
        }
        a = find_root(parent, a, status, ctl);
        b = find_root(parent, b, status, ctl);
        if (a == b) break;
        if (a < b) {
          const i32 t = a;
          a = b;
          b = t;
        }
        if (atomicCAS(&parent[a], a, b) == a) break;
      }
    }
    barrier(g);
  }
  for (i64 e = tid; e < E; e += nth)
    if (mst[e] == MST_DROPPED) mst[e] = 0;
  // labels: the root, which is the smallest vertex of its component
  long long roots = 0;
  for (i64 v = tid; v < n; v += nth) {
    const i32 r = find_root(parent, (i32)v, status, ctl);
    comp[v] = r;
    roots += (r == (i32)v);
  }
  for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(0xffffffffu, roots, o);
  if ((threadIdx.x & 31) == 0 && roots) atomicAdd((unsigned long long*)&ctl->ncomp, (unsigned long long)roots);
}

// Cluster form for small and medium graphs: one cluster of 8 or 16 blocks,
// whose barriers cost a fraction of a grid barrier, three barriers a round.
// Offers: every edge between two components offers (rank << 32 | the other
// root) to both roots with a 64-bit atomicMin, so the winning word names the
// chosen edge and the component across it. Hooks: every root with an offer
// marks the edge and points to the other root; of a mutual pair only the
// larger root hooks, so no cycle can form. Flatten: all vertices halve their
// paths at once, so the hook trees collapse in a logarithmic number of steps
// and the next round's offers read roots with one load. Offer words alternate
// between two arrays by round, the idle one being cleared during the hooks.
// Parents and offers live in global memory: scattered single-word accesses
// from many blocks are served by the L2 slices in parallel.
constexpr int MSTC_NT = 512;
constexpr int MSTC_B = 2;  // edges per thread and batch (2 walks each)
constexpr u64 NO_OFFER = ~0ull;

// path halving of K vertices in lockstep (their loads overlap); leaves each
// vertex pointing at its root; slots < 0 are padding
template <int K>
__device__ __forceinline__ void halve_many(volatile i32* par, const i32 (&v)[K], int* bad) {
  i32 x[K];
#pragma unroll
  for (int k = 0; k < K; ++k) x[k] = v[k];
  for (int it = 0; it < (1 << 20); ++it) {
    i32 p[K], gp[K];
#pragma unroll
    for (int k = 0; k < K; ++k) p[k] = x[k] >= 0 ? par[x[k]] : -1;
#pragma unroll
    for (int k = 0; k < K; ++k) gp[k] = p[k] >= 0 ? par[p[k]] : -1;
    bool moved = false;
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (gp[k] != p[k]) {
        par[x[k]] = gp[k];
        x[k] = gp[k];
        moved = true;
      }
    if (!moved) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (v[k] >= 0 && p[k] != v[k]) par[v[k]] = p[k];
      return;
    }
  }
  *bad = 1;
}

__global__ void __launch_bounds__(MSTC_NT, 1) k_mst_cluster(const i32* __restrict__ ei, const i32* __restrict__ ej,
                                                            i64 E, i64 n, i32* par_g, u64* offer, i32* minv,
                                                            uint8_t* __restrict__ mst, i32* __restrict__ comp,
                                                            MstCtl* ctl, int* status, int max_rounds) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ int flag[2];  // rank 0's words: bit 0 some offer this round, bit 1 a loop bound was hit
  __shared__ int bad;
  cg::cluster_group cl = cg::this_cluster();
  const int cs = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const int tid = threadIdx.x;
  const i64 gtid = (i64)rank * MSTC_NT + tid, gs = (i64)cs * MSTC_NT;
  volatile i32* par = par_g;
  volatile u64* voff = offer;
  for (i64 v = gtid; v < n; v += gs) {
    par[v] = (i32)v;
    offer[v] = NO_OFFER;
    offer[n + v] = NO_OFFER;
    minv[v] = INT_MAX;
  }
  for (i64 e = gtid; e < E; e += gs) mst[e] = 0;
  if (tid == 0) {
    flag[0] = 0;
    flag[1] = 0;
    bad = 0;
    if (rank == 0) ctl->ncomp = 0;
  }
  int* flag0 = cl.map_shared_rank(flag, 0u);
  cl.sync();
  for (int round = 0;; ++round) {
    if (round >= max_rounds) {
      if (gtid == 0) set_status(status, PH_ERR_ITER_LIMIT);
      break;
    }
    u64* cur = offer + (size_t)(round & 1) * n;
    volatile u64* vcur = voff + (size_t)(round & 1) * n;
    bool offered = false;
    for (i64 e0 = gtid; e0 < E; e0 += gs * MSTC_B) {
      i32 x[2 * MSTC_B];
#pragma unroll
      for (int k = 0; k < MSTC_B; ++k) {
        const i64 e = e0 + k * gs;
        x[2 * k] = e < E ? __ldg(ei + e) : -1;
        x[2 * k + 1] = e < E ? __ldg(ej + e) : -1;
      }
#pragma unroll
      for (int k = 0; k < 2 * MSTC_B; ++k) x[k] = x[k] >= 0 ? par[x[k]] : -1;  // parents are flat here
      u64 ou[MSTC_B], ov[MSTC_B];
#pragma unroll
      for (int k = 0; k < MSTC_B; ++k)
        if (x[2 * k] != x[2 * k + 1]) {
          ou[k] = vcur[x[2 * k]];
          ov[k] = vcur[x[2 * k + 1]];
        }
#pragma unroll
      for (int k = 0; k < MSTC_B; ++k) {
        const i32 ru = x[2 * k], rv = x[2 * k + 1];
        if (ru == rv) continue;  // also the padding slots (-1, -1)
        const u64 e = (u64)(e0 + k * gs);
        const u64 wu = (e << 32) | (u32)rv, wv = (e << 32) | (u32)ru;
        // a read first: most offers to a busy root lose to a smaller one
        if (wu < ou[k]) atomicMin((unsigned long long*)&cur[ru], (unsigned long long)wu);
        if (wv < ov[k]) atomicMin((unsigned long long*)&cur[rv], (unsigned long long)wv);
        offered = true;
      }
    }
    // every block leaves the loop in the same round
    const int f = __syncthreads_or(offered) ? 1 : 0;
    if (tid == 0 && (f | *(volatile int*)&bad)) atomicOr(flag0 + (round & 1), f | (*(volatile int*)&bad ? 2 : 0));
    cl.sync();
    const int word = *(volatile int*)(flag0 + (round & 1));
    if (word != 1) break;
    // the other word is next read after the barrier below
    if (rank == 0 && tid == 0) flag[(round + 1) & 1] = 0;
    // hooks; the other offer array (last read in the previous round) is cleared
    u64* idle = offer + (size_t)((round + 1) & 1) * n;
    for (i64 v = gtid; v < n; v += gs) {
      idle[v] = NO_OFFER;
      const u64 w = vcur[v];
      if (w == NO_OFFER) continue;
      const i32 e = (i32)(w >> 32), o = (i32)(w & 0xffffffffull);
      mst[e] = 1;
      if ((vcur[o] >> 32) == (u64)e && o > (i32)v) continue;  // mutual choice: the larger root hooks
      par[v] = o;
    }
    cl.sync();
    // flatten: every vertex halves its path at the same time, so the depth of
    // the hook trees falls geometrically and the next offers read roots directly
    for (i64 v0 = gtid; v0 < n; v0 += gs * MSTC_B) {
      i32 x[MSTC_B];
#pragma unroll
      for (int k = 0; k < MSTC_B; ++k) x[k] = v0 + k * gs < n ? (i32)(v0 + k * gs) : -1;
      halve_many(par, x, &bad);
    }
    cl.sync();
  }
  // labels: the smallest vertex of each component, and the component count
  unsigned long long roots = 0;
  for (i64 v = gtid; v < n; v += gs) {
    const i32 r = par[v];  // flat after the last round's flatten
    atomicMin(minv + r, (i32)v);
    roots += (r == (i32)v);
  }
  for (int o = 16; o > 0; o >>= 1) roots += __shfl_xor_sync(0xffffffffu, roots, o);
  if ((tid & 31) == 0 && roots) atomicAdd((unsigned long long*)&ctl->ncomp, roots);
  cl.sync();
  for (i64 v = gtid; v < n; v += gs) comp[v] = minv[par[v]];
  if (*(volatile int*)&bad && tid == 0) set_status(status, PH_ERR_ITER_LIMIT);
  cl.sync();  // rank 0's flag words stay valid until every block is done with them
}

__global__ void k_copy_ncomp(const MstCtl* ctl, int64_t* out) {
  ph::pdl_wait();
  ph::pdl_trigger(); *out = ctl->ncomp; }

__global__ void k_h0_rows(const float* __restrict__ filt, const uint8_t* __restrict__ mst,
                          const i32* __restrict__ pos, i64 E, i64 n, float* __restrict__ rows) {
  ph::pdl_wait();
  ph::pdl_trigger();
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

// Cluster size of the cluster form on the current device (16 where a 16-block
// cluster of this kernel can be resident, else 8, 0 when neither can). The
// function attribute belongs to a device, so it is set, and the answer
// cached, once per device.
int cluster_size() {
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
  cudaFuncSetAttribute((const void*)k_mst_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (int cs : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(MSTC_NT);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)k_mst_cluster, &cfg) == cudaSuccess && clusters > 0) {
      cached[dev] = cs;
      break;
    }
  }
  cudaGetLastError();
  return cached[dev];
}

extern "C" size_t ph_boruvka_workspace_bytes(int64_t n, int64_t E) {
  (void)E;
  // parents and offers (grid form); parents, two offer arrays and labels (cluster form)
  return 2 * Carve::need((size_t)n * 4) + Carve::need(sizeof(MstCtl)) + Carve::need((size_t)n * 16) +
         Carve::need((size_t)n * 4);
}

extern "C" int ph_boruvka_mst(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                              uint8_t* mst_mask, int32_t* comp, int64_t* d_ncomp, int* d_status,
                              void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || E < 0 || n >= (int64_t(1) << 31) || E >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  if (n == 0) {
    ph::zero_async(d_ncomp, sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  i32* parent = c.take<i32>(n);
  i32* best = c.take<i32>(n);
  MstCtl* ctl = c.take<MstCtl>(1);
  u64* offer = c.take<u64>(2 * n);
  i32* minv = c.take<i32>(n);
  if (!parent || !best || !ctl || !offer || !minv) return PH_ERR_ARG;
  const i64 work = std::max<i64>(n, E);
  int max_rounds = 2;
  while ((i64(1) << (max_rounds - 2)) < n && max_rounds < 64) ++max_rounds;
  max_rounds += 4;
  const int cs = work > 4096 && work <= (i64(1) << 18) ? cluster_size() : 0;
  if (cs > 0) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(MSTC_NT);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    ph::count_launch();
    if (cudaLaunchKernelEx(&cfg, k_mst_cluster, edge_i, edge_j, (i64)E, (i64)n, parent, offer, minv, mst_mask, comp,
                           ctl, d_status, max_rounds) != cudaSuccess)
      return PH_ERR_CUDA;
  } else if (work <= 4 * MST_NT * 8) {
    ph::count_launch();
    ph::launch_pdl(k_mst, dim3(1), dim3(MST_NT), 0, s, edge_i, edge_j, E, n, parent, best, mst_mask, comp, ctl, d_status, max_rounds);
  } else {
    const int sms = ph::device_sms();
    const int per_sm = ph::occupancy((const void*)k_mst, MST_NT, 0);
    if (per_sm < 1) return PH_ERR_CUDA;
    const i64 want = (work + MST_NT * 2 - 1) / (MST_NT * 2);
    const int blocks = (int)std::max<i64>(2, std::min<i64>(want, (i64)sms * per_sm));
    void* args[] = {(void*)&edge_i, (void*)&edge_j,   (void*)&E,    (void*)&n,   (void*)&parent,
                    (void*)&best,   (void*)&mst_mask, (void*)&comp, (void*)&ctl, (void*)&d_status,
                    (void*)&max_rounds};
    ph::count_launch();
    if (cudaLaunchCooperativeKernel((const void*)k_mst, blocks, MST_NT, args, 0, s) != cudaSuccess)
      return PH_ERR_CUDA;
  }
  ph::count_launch();
  ph::launch_pdl(k_copy_ncomp, dim3(1), dim3(1), 0, s, ctl, d_ncomp);
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
  ph::launch_pdl(k_h0_rows, dim3(g), dim3(256), 0, s, edge_filt, mst_mask, pos, E, n, out_rows);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
