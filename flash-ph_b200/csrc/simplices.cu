// Triangles and tetrahedra of the Rips complex, emitted directly in
// filtration order, and the cofacet (coboundary) CSR built from them.
//
// Reference: triangle_kernel.py:28-144,152-270,288-505 (enumeration),
// reduce_h1_gpu.py:65-152,509-521 (face ranks, triangle order, cofacet CSR).
//
// The reference enumerates triangles per edge (third vertex above both
// endpoints), then looks up face ranks with a sort + searchsorted and orders
// the triangles with two stable argsorts by (largest edge rank, colex). Here
// every triangle is generated from its largest edge m = (a, b): its third
// vertex w is a common neighbour of a and b with both other edges ranked
// below m. For a fixed largest edge the colex order of {a, b, w} is the order
// of w, so walking w upward per m yields the reference's (max_rank, colex)
// order with no sort, and the face ranks fall out of the adjacency walk.
// Tetrahedra are generated the same way from their largest edge m: pairs
// p < q of third vertices of m's triangles whose edge (p, q) ranks below m.
// One warp handles one edge: lanes take 32 consecutive entries of the shorter
// adjacency row and binary-search the longer one; ballots keep the output in
// order.
#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int SX_NT = 256;
constexpr int SX_WARPS = SX_NT / 32;
// Entries of an adjacency row a warp copies into its shared memory before
// searching it many times (dense graphs: rows of a few hundred entries,
// searched by every candidate of the other row): a search then costs shared-
// memory latency per step instead of a dependent global load. 8 warps x 576
// entries x (index, rank) = 36 KB a block.
constexpr int SX_STAGE = 576;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int lower_bound_i32(const i32* __restrict__ a, int lo, int hi, i32 x) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// EMIT = false: count; EMIT = true: write triangles.
template <bool EMIT>
__global__ void __launch_bounds__(SX_NT) k_triangles(const i32* __restrict__ ei, const i32* __restrict__ ej,
                                                    i64 E, const i32* __restrict__ aptr,
                                                    const i32* __restrict__ aidx,
                                                    const i32* __restrict__ arank,
                                                    i32* __restrict__ tri_cnt, i32* __restrict__ cof_cnt,
                                                    const i64* __restrict__ tri_off, i32* __restrict__ tm,
                                                    i32* __restrict__ tw, i32* __restrict__ tfa,
                                                    i32* __restrict__ tfb, const uint8_t* __restrict__ keep,
                                                    const i32* __restrict__ vcloud) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ i32 st_idx[SX_WARPS][SX_STAGE];
  __shared__ i32 st_rank[SX_WARPS][SX_STAGE];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const i64 warp = ((i64)blockIdx.x * SX_NT + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * SX_NT) >> 5;
  const u32 lt = lanemask_lt();
  for (i64 m = warp; m < E; m += nwarps) {
    __syncwarp();  // the previous edge's searches of the staged row are done
    const i32 a = ei[m], b = ej[m];
    // a batch's count pass: the edges of a cloud already over its limit count nothing
    if (keep && !keep[vcloud[a]]) {
      if (!EMIT && lane == 0) {
        tri_cnt[m] = 0;
        cof_cnt[m] = 0;
      }
      continue;
    }
    int sa = aptr[a], ea = aptr[a + 1], sb = aptr[b], eb = aptr[b + 1];
    // walk the shorter row, search the longer
    const bool a_short = (ea - sa) <= (eb - sb);
    const int s0 = a_short ? sa : sb, s1 = a_short ? ea : eb;
    const int l0 = a_short ? sb : sa, l1 = a_short ? eb : ea;
    int ntri = 0, ncof = 0;
    i64 out = EMIT ? tri_off[m] : 0;
    // the emit pass writes only inside the edge's allotment [tri_off[m],
    // tri_off[m + 1]): an edge allotted nothing (a batch can clear the
    // triangles of some clouds after the count) is skipped
    const i64 oend = EMIT ? tri_off[m + 1] : 0;
    if (EMIT && oend <= out) continue;
    // a long row searched by more than one round of lanes is staged first
    const int nl = l1 - l0;
    const bool staged = nl > 32 && nl <= SX_STAGE && s1 - s0 > 32;
    if (staged) {
      for (int k = lane; k < nl; k += 32) {
        st_idx[wl][k] = aidx[l0 + k];
        st_rank[wl][k] = arank[l0 + k];
      }
      __syncwarp();
    }
    for (int base = s0; base < s1; base += 32) {
      const int p = base + lane;
      bool common = false, valid = false;
      i32 w = 0, rs = 0, rl = 0;
      if (p < s1) {
        w = aidx[p];
        rs = arank[p];
        if (staged) {
          const int q = lower_bound_i32(st_idx[wl], 0, nl, w);
          if (q < nl && st_idx[wl][q] == w) {
            common = true;
            rl = st_rank[wl][q];
            valid = rs < (i32)m && rl < (i32)m;
          }
        } else {
          const int q = lower_bound_i32(aidx, l0, l1, w);
          if (q < l1 && aidx[q] == w) {
            common = true;
            rl = arank[q];
            valid = rs < (i32)m && rl < (i32)m;
          }
        }
      }
      const u32 cb = __ballot_sync(FULL, common);
      const u32 vb = __ballot_sync(FULL, valid);
      if (EMIT && valid && out + __popc(vb & lt) < oend) {
        const i64 o = out + __popc(vb & lt);
        tm[o] = (i32)m;
        tw[o] = w;
        tfa[o] = a_short ? rs : rl;  // rank of (a, w)
        tfb[o] = a_short ? rl : rs;  // rank of (b, w)
      }
      ncof += __popc(cb);
      ntri += __popc(vb);
      out += __popc(vb);
    }
    if (!EMIT && lane == 0) {
      tri_cnt[m] = ntri;
      cof_cnt[m] = ncof;
    }
  }
}

// Exact number of triangles of the graph (each counted once, at its smallest
// vertex x and middle vertex y: pairs x < y < z, all three edges present).
// One CTA per vertex a (persistent over vertices): N(a) goes into a shared
// bitmap, each warp takes a neighbour b > a and tests its neighbours w > b
// against the bitmap. No ranks are needed, since every triangle has exactly
// one largest edge; the result equals the sum of the per-edge triangle counts.
// UPPER: the rows hold only the larger neighbours, in any order (the upper
// adjacency of k_upper_fill), so no row is searched; otherwise the rows are
// the full adjacency sorted by neighbour.
// SEG: per-cloud totals of a batch's union graph: vertex a counts into
// per[vcloud[a]], and only the vertices of clouds with want[cloud] set are
// visited (total unused).
template <bool UPPER, bool SEG = false>
__global__ void __launch_bounds__(SX_NT) k_tri_total(const i32* __restrict__ aptr, const i32* __restrict__ aidx,
                                                    i64 n, int* __restrict__ next,
                                                    unsigned long long* __restrict__ total,
                                                    const i32* __restrict__ vcloud = nullptr,
                                                    const uint8_t* __restrict__ want = nullptr,
                                                    unsigned long long* __restrict__ per = nullptr) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ u32 nbits[];
  __shared__ int cur;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const i64 words = (n + 31) >> 5;
  for (i64 w = threadIdx.x; w < words; w += SX_NT) nbits[w] = 0u;
  unsigned long long cnt = 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) cur = atomicAdd(next, 1);
    __syncthreads();
    const i64 a = cur;
    if (a >= n) break;
    if (SEG && !want[vcloud[a]]) continue;
    const int s = aptr[a], e = aptr[a + 1];
    if (e - s < 2) continue;
    for (int p = s + threadIdx.x; p < e; p += SX_NT) {
      const i32 v = aidx[p];
      atomicOr(&nbits[v >> 5], 1u << (v & 31));
    }
    __syncthreads();
    // neighbours b > a of a (sorted rows: from the first one above a)
    const int first = UPPER ? s : lower_bound_i32(aidx, s, e, (i32)a + 1);
    for (int p = first + warp; p < e; p += SX_NT / 32) {
      const i32 b = aidx[p];
      const int sb = aptr[b], eb = aptr[b + 1];
      for (int q = (UPPER ? sb : lower_bound_i32(aidx, sb, eb, b + 1)) + lane; q < eb; q += 32) {
        const i32 w = aidx[q];
        cnt += (nbits[w >> 5] >> (w & 31)) & 1u;
      }
    }
    __syncthreads();
    for (int p = s + threadIdx.x; p < e; p += SX_NT) {
      const i32 v = aidx[p];
      nbits[v >> 5] = 0u;
    }
    if (SEG) {  // this vertex's triangles to its cloud
      for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(FULL, cnt, o);
      if (lane == 0 && cnt) atomicAdd(per + vcloud[a], cnt);
      cnt = 0;
    }
  }
  if (SEG) return;
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(FULL, cnt, o);
  if (lane == 0 && cnt) atomicAdd(total, cnt);
}

// upper adjacency of unsorted edges i < j: row i lists every j, in any order
__global__ void k_upper_deg(const i32* __restrict__ ei, i64 E, i32* __restrict__ deg) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x)
    atomicAdd(&deg[ei[e]], 1);
}

__global__ void k_upper_fill(const i32* __restrict__ ei, const i32* __restrict__ ej, i64 E,
                             const i32* __restrict__ uptr, i32* __restrict__ cursor, i32* __restrict__ uidx) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (i64)gridDim.x * blockDim.x) {
    const i32 i = ei[e];
    uidx[uptr[i] + atomicAdd(&cursor[i], 1)] = ej[e];
  }
}

// Tetrahedra with largest edge m: pairs (i < k) of m's triangles whose third
// vertices p = W[i], q = W[k] are joined by an edge ranked below m.
template <bool EMIT>
__global__ void __launch_bounds__(SX_NT) k_tets(const i32* __restrict__ ei, const i32* __restrict__ ej, i64 E,
                                               const i64* __restrict__ tri_off, const i32* __restrict__ tw,
                                               const i32* __restrict__ tfa, const i32* __restrict__ tfb,
                                               const i32* __restrict__ aptr, const i32* __restrict__ aidx,
                                               const i32* __restrict__ arank, const uint8_t* __restrict__ enable,
                                               i32* __restrict__ tet_cnt, const i64* __restrict__ tet_off,
                                               i32* __restrict__ qm, i32* __restrict__ qf, int* status) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ i32 st_idx[SX_WARPS][SX_STAGE];
  __shared__ i32 st_rank[SX_WARPS][SX_STAGE];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const i64 warp = ((i64)blockIdx.x * SX_NT + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * SX_NT) >> 5;
  const u32 lt = lanemask_lt();
  for (i64 m = warp; m < E; m += nwarps) {
    const i64 t0 = tri_off[m], t1 = tri_off[m + 1];
    const int nw = (enable && !enable[m]) ? 0 : (int)(t1 - t0);
    i64 out = EMIT ? tet_off[m] : 0;
    const i64 oend = EMIT ? tet_off[m + 1] : 0;  // writes stay inside the edge's allotment
    int cnt = 0;
    for (int i = 0; i + 1 < nw; ++i) {
      const i32 p = tw[t0 + i];
      const int sp = aptr[p], ep = aptr[p + 1];
      // N(p) searched by more than one round of lanes: staged first
      const int np = ep - sp;
      const bool staged = np > 32 && np <= SX_STAGE && nw - i - 1 > 32;
      __syncwarp();  // the previous searches of the staged row are done
      if (staged) {
        for (int k = lane; k < np; k += 32) {
          st_idx[wl][k] = aidx[sp + k];
          st_rank[wl][k] = arank[sp + k];
        }
        __syncwarp();
      }
      for (int kb = i + 1; kb < nw; kb += 32) {
        const int k = kb + lane;
        bool valid = false;
        i32 q = 0, rpq = 0;
        if (k < nw) {
          q = tw[t0 + k];
          if (staged) {
            const int pos = lower_bound_i32(st_idx[wl], 0, np, q);
            if (pos < np && st_idx[wl][pos] == q) {
              rpq = st_rank[wl][pos];
              valid = rpq < (i32)m;
            }
          } else {
            const int pos = lower_bound_i32(aidx, sp, ep, q);
            if (pos < ep && aidx[pos] == q) {
              rpq = arank[pos];
              valid = rpq < (i32)m;
            }
          }
        }
        const u32 vb = __ballot_sync(FULL, valid);
        if (EMIT && valid && out + __popc(vb & lt) < oend) {
          const i64 o = out + __popc(vb & lt);
          qm[o] = (i32)m;
          qf[4 * o + 0] = (i32)(t0 + i);
          qf[4 * o + 1] = (i32)(t0 + k);
          // faces {a, p, q} and {b, p, q}: find their largest edge and third vertex
          const i32 a = ei[m], b = ej[m];
#pragma unroll
          for (int side = 0; side < 2; ++side) {
            const i32 x = side ? b : a;
            const i32 rxp = side ? tfb[t0 + i] : tfa[t0 + i];
            const i32 rxq = side ? tfb[t0 + k] : tfa[t0 + k];
            i32 M, third;
            if (rxp > rxq && rxp > rpq) {
              M = rxp;
              third = q;
            } else if (rxq > rpq) {
              M = rxq;
              third = p;
            } else {
              M = rpq;
              third = x;
            }
            const int lo = (int)tri_off[M], hi = (int)tri_off[M + 1];
            int f = lower_bound_i32(tw, lo, hi, third);
            if (f >= hi || tw[f] != third) {  // cannot happen for a consistent adjacency
              set_status(status, PH_ERR_ARG);
              f = (int)t0;
            }
            qf[4 * o + 2 + side] = f;
          }
        }
        cnt += __popc(vb);
        out += __popc(vb);
      }
    }
    if (!EMIT && lane == 0) tet_cnt[m] = cnt;
  }
}

// Cofacet entries (face, simplex rank) in ascending simplex order.
__global__ void k_cof_entries(const i32* __restrict__ faos, const i32* __restrict__ f0,
                              const i32* __restrict__ f1, const i32* __restrict__ f2, int k, i64 S,
                              i32 row_base, u64* __restrict__ keys, u32* __restrict__ vals) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const i64 total = S * k;
  for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (i64)gridDim.x * blockDim.x) {
    const i64 s = x / k;
    const int z = (int)(x - s * k);
    i32 f;
    if (faos) f = faos[x];
    else f = z == 0 ? f0[s] : (z == 1 ? f1[s] : f2[s]);
    keys[x] = (u64)(u32)f;
    vals[x] = (u32)(row_base + s);
  }
}

__global__ void k_cof_fill(const u64* __restrict__ keys, const u32* __restrict__ vals, i64 H, i64 nf,
                           i32* __restrict__ off, i32* __restrict__ data) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x; p < H; p += (i64)gridDim.x * blockDim.x) {
    const i64 f = (i64)keys[p];
    data[p] = (i32)vals[p];
    const i64 prev = p ? (i64)keys[p - 1] : -1;
    for (i64 v = prev + 1; v <= f; ++v) off[v] = (i32)p;
    if (p == H - 1)
      for (i64 v = f + 1; v <= nf; ++v) off[v] = (i32)H;
  }
}

__global__ void k_cmf(const i32* __restrict__ faos, const i32* __restrict__ f0, const i32* __restrict__ f1,
                      const i32* __restrict__ f2, int k, i64 S, i32 face_base,
                      const uint8_t* __restrict__ skip, i32* __restrict__ cmf) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 s = (i64)blockIdx.x * blockDim.x + threadIdx.x; s < S; s += (i64)gridDim.x * blockDim.x) {
    i32 best = -1;
    for (int z = 0; z < k; ++z) {
      i32 f;
      if (faos) f = faos[s * k + z];
      else f = z == 0 ? f0[s] : (z == 1 ? f1[s] : f2[s]);
      if (!skip[f]) best = max(best, face_base + f);
    }
    cmf[s] = best;
  }
}

// ---- cofacet rows without a global sort -----------------------------------------------
// The H1 cofacet rows are known in length before any triangle is stored: the
// row of edge e holds every triangle containing e, one per common neighbour
// of its ends, which the triangle count pass counts (cof_off). So the entries
// can be scattered straight into their rows (an atomic cursor per row), and
// only each row needs ordering: a warp sorts a row of up to 1024 entries
// (a bitonic network in registers for <= 32, in the warp's shared memory
// above), a block the rows up to RS_BIG entries. This replaces the stable
// radix sort of all 3T entries by face, whose passes dominate dense batches.
constexpr int RS_WARP_MAX = 1024;        // entries a warp sorts in shared memory
constexpr int RS_BIG = 8192;             // entries a block sorts in shared memory
static_assert(RS_BIG == ph::COF_ROWS_MAX, "the callers' row bound is the block sort's size");
constexpr int RS_NT = 256;

__global__ void k_off_i64_to_i32(const i64* __restrict__ in, i64 n, i32* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (i64)gridDim.x * blockDim.x)
    out[i] = (i32)in[i];
}

// every triangle's rank into the rows of its three faces; a write past its
// row's end (counts inconsistent with the triangles) is dropped and reported
__global__ void k_cof_scatter3(const i32* __restrict__ f0, const i32* __restrict__ f1, const i32* __restrict__ f2,
                               i64 S, i32 row_base, const i32* __restrict__ off, i32* __restrict__ cursor,
                               i32* __restrict__ data, int* status) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 s = (i64)blockIdx.x * blockDim.x + threadIdx.x; s < S; s += (i64)gridDim.x * blockDim.x) {
    const i32 r = row_base + (i32)s;
    const i32 f[3] = {f0[s], f1[s], f2[s]};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const i32 pos = off[f[q]] + atomicAdd(&cursor[f[q]], 1);
      if (pos < off[f[q] + 1]) data[pos] = r;
      else set_status(status, PH_ERR_ARG);
    }
  }
}

// the cofacet rows of k-simplices given as k faces each (AoS): the row
// lengths first (a count per face), then each simplex's rank into its faces'
// rows; a write past its row's end is dropped and reported
__global__ void k_cof_count_aos(const i32* __restrict__ faos, i64 H, i32* __restrict__ cnt) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < H; x += (i64)gridDim.x * blockDim.x)
    atomicAdd(&cnt[faos[x]], 1);
}

__global__ void k_cof_scatter_aos(const i32* __restrict__ faos, i64 H, int k, i32 row_base,
                                  const i32* __restrict__ off, i32* __restrict__ cursor, i32* __restrict__ data,
                                  int* status) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < H; x += (i64)gridDim.x * blockDim.x) {
    const i32 f = faos[x];
    const i32 pos = off[f] + atomicAdd(&cursor[f], 1);
    if (pos < off[f + 1]) data[pos] = row_base + (i32)(x / k);
    else set_status(status, PH_ERR_ARG);
  }
}

// ascending bitonic sort of n <= len2 (a power of two) values in shared memory
// by the threads tid = 0..nthreads-1 of a group that synchronises with sync()
template <typename Sync>
__device__ __forceinline__ void bitonic_shared(i32* v, int len2, int tid, int nthreads, Sync sync) {
  for (int size = 2; size <= len2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < (len2 >> 1); i += nthreads) {
        const int lo = 2 * i - (i & (stride - 1));  // index with bit `stride` clear
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const i32 x = v[lo], y = v[hi];
        if ((x > y) == up) {
          v[lo] = y;
          v[hi] = x;
        }
      }
      sync();
    }
  }
}

// rows of up to RS_WARP_MAX entries: one warp a row; longer rows are listed
// (up to RS_BIG entries) for k_cof_sort_big
__global__ void __launch_bounds__(RS_NT) k_cof_sort_rows(const i32* __restrict__ off, i64 nrows,
                                                         i32* __restrict__ data, i32* __restrict__ big,
                                                         int* __restrict__ nbig) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ i32 buf[RS_NT / 32][RS_WARP_MAX];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const i64 warp = ((i64)blockIdx.x * RS_NT + threadIdx.x) >> 5;
  const i64 nwarps = ((i64)gridDim.x * RS_NT) >> 5;
  for (i64 r = warp; r < nrows; r += nwarps) {
    const i32 o = off[r];
    const int len = off[r + 1] - o;
    if (len <= 1) continue;
    if (len <= 32) {
      // bitonic network across the lanes (pads sort last)
      i32 x = lane < len ? data[o + lane] : INT_MAX;
      for (int size = 2; size <= 32; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          const i32 y = __shfl_xor_sync(0xffffffffu, x, stride);
          const bool up = (lane & size) == 0;
          const bool lower = (lane & stride) == 0;
          x = (lower == up) ? min(x, y) : max(x, y);
        }
      }
      if (lane < len) data[o + lane] = x;
      continue;
    }
    if (len > RS_WARP_MAX) {
      if (lane == 0) big[atomicAdd(nbig, 1)] = (i32)r;
      continue;
    }
    int len2 = 64;
    while (len2 < len) len2 <<= 1;
    __syncwarp();
    for (int i = lane; i < len2; i += 32) buf[wl][i] = i < len ? data[o + i] : INT_MAX;
    __syncwarp();
    bitonic_shared(buf[wl], len2, lane, 32, []() { __syncwarp(); });
    for (int i = lane; i < len; i += 32) data[o + i] = buf[wl][i];
    __syncwarp();
  }
}

// the listed long rows, one block a row
__global__ void __launch_bounds__(RS_NT) k_cof_sort_big(const i32* __restrict__ off, i32* __restrict__ data,
                                                        const i32* __restrict__ big, const int* __restrict__ nbig,
                                                        int* status) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ i32 buf[RS_BIG];
  const int nb = *nbig;
  for (int q = blockIdx.x; q < nb; q += gridDim.x) {
    const i32 r = big[q];
    const i32 o = off[r];
    const int len = off[r + 1] - o;
    if (len > RS_BIG) {  // the caller checked the longest row; a longer one means inconsistent inputs
      if (threadIdx.x == 0) set_status(status, PH_ERR_ARG);
      continue;
    }
    int len2 = 2 * RS_WARP_MAX;
    while (len2 < len) len2 <<= 1;
    __syncthreads();
    for (int i = threadIdx.x; i < len2; i += RS_NT) buf[i] = i < len ? data[o + i] : INT_MAX;
    __syncthreads();
    bitonic_shared(buf, len2, threadIdx.x, RS_NT, []() { __syncthreads(); });
    for (int i = threadIdx.x; i < len; i += RS_NT) data[o + i] = buf[i];
  }
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}
inline int warp_grid(i64 items) {
  return (int)std::max<i64>(1, std::min<i64>((items * 32 + SX_NT - 1) / SX_NT, 148 * 32));
}

}  // namespace
}  // namespace ph

using namespace ph;

extern "C" size_t ph_triangles_count_workspace_bytes(int64_t E) {
  return 2 * Carve::need((size_t)(E + 1) * 4) + scan_workspace_bytes(E);
}

extern "C" int ph_triangles_count(const int32_t* edge_i, const int32_t* edge_j, int64_t E,
                                  const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                                  int64_t* tri_off, int64_t* cof_off, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  return ph::triangles_count_masked(edge_i, edge_j, E, adj_ptr, adj_idx, adj_rank, tri_off, cof_off, workspace,
                                    workspace_bytes, nullptr, nullptr, (cudaStream_t)stream);
}

// The count pass with an optional per-cloud mask (keep[vcloud[i]] == 0: the
// edge counts nothing), for a batch whose over-limit clouds are known first.
int ph::triangles_count_masked(const int32_t* edge_i, const int32_t* edge_j, int64_t E, const int32_t* adj_ptr,
                               const int32_t* adj_idx, const int32_t* adj_rank, int64_t* tri_off, int64_t* cof_off,
                               void* workspace, size_t workspace_bytes, const uint8_t* keep, const int32_t* vcloud,
                               cudaStream_t s) {
  if (E < 0) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  i32* tc = c.take<i32>(E + 1);
  i32* cc = c.take<i32>(E + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(E));
  if (!tc || !cc || !sws) return PH_ERR_ARG;
  if (E > 0) {
    ph::count_launch();
    ph::launch_pdl(k_triangles<false>, dim3(warp_grid(E)), dim3(SX_NT), 0, s, edge_i, edge_j, E, adj_ptr, adj_idx, adj_rank, tc, cc,
                                                      nullptr, nullptr, nullptr, nullptr, nullptr, keep, vcloud);
  }
  PH_TRY(scan_exclusive_i32_i64(tc, tri_off, E, sws, scan_workspace_bytes(E), s));
  PH_TRY(scan_exclusive_i32_i64(cc, cof_off, E, sws, scan_workspace_bytes(E), s));
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int64_t ph_triangles_total_max_vertices(void) { return (int64_t)(200 * 1024) * 8; }

extern "C" int ph_triangles_total(const int32_t* adj_ptr, const int32_t* adj_idx, int64_t n,
                                  unsigned long long* d_total, int* d_next, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !d_total || !d_next) return PH_ERR_ARG;
  if (n > ph_triangles_total_max_vertices()) {
    record_message("ph_triangles_total: n exceeds the shared-memory bitmap (1638400 vertices)");
    return PH_ERR_ARG;
  }
  ph::zero_async(d_total, sizeof(unsigned long long), s, d_next, sizeof(int));
  if (n < 3) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  const size_t smem = (size_t)((n + 31) / 32) * 4;
  if (smem > 48 * 1024 && ph::allow_dynamic_smem((const void*)k_tri_total<false>) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  const int sms = ph::device_sms();
  const int occ = ph::occupancy((const void*)k_tri_total<false>, SX_NT, smem);
  const int grid = (int)std::max<i64>(1, std::min<i64>(n, (i64)sms * std::max(occ, 1)));
  ph::count_launch();
  ph::launch_pdl(k_tri_total<false>, dim3(grid), dim3(SX_NT), smem, s, adj_ptr, adj_idx, n, d_next, d_total,
                 (const i32*)nullptr, (const uint8_t*)nullptr, (unsigned long long*)nullptr);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_batch_triangles_total(const int32_t* adj_ptr, const int32_t* adj_idx, int64_t n,
                                        const int32_t* vcloud, const uint8_t* want, int32_t nclouds,
                                        unsigned long long* d_per, int* d_next, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || nclouds < 1 || !adj_ptr || !vcloud || !want || !d_per || !d_next) return PH_ERR_ARG;
  if (n > ph_triangles_total_max_vertices()) {
    record_message("ph_batch_triangles_total: n exceeds the shared-memory bitmap (1638400 vertices)");
    return PH_ERR_ARG;
  }
  ph::zero_async(d_per, sizeof(unsigned long long) * (size_t)nclouds, s, d_next, sizeof(int));
  if (n < 3) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  const size_t smem = (size_t)((n + 31) / 32) * 4;
  if (smem > 48 * 1024 && ph::allow_dynamic_smem((const void*)k_tri_total<false, true>) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  const int sms = ph::device_sms();
  const int occ = ph::occupancy((const void*)k_tri_total<false, true>, SX_NT, smem);
  const int grid = (int)std::max<i64>(1, std::min<i64>(n, (i64)sms * std::max(occ, 1)));
  ph::count_launch();
  ph::launch_pdl(k_tri_total<false, true>, dim3(grid), dim3(SX_NT), smem, s, adj_ptr, adj_idx, n, d_next,
                 (unsigned long long*)nullptr, vcloud, want, d_per);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_triangles_total_edges_workspace_bytes(int64_t E, int64_t n) {
  return Carve::need(sizeof(i32) * (size_t)(n + 1)) * 3 + Carve::need(sizeof(i32) * (size_t)std::max<i64>(E, 1)) +
         Carve::need(scan_workspace_bytes(n)) + Carve::need(sizeof(int));
}

extern "C" int ph_triangles_total_edges(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                                        unsigned long long* d_total, void* workspace, size_t workspace_bytes,
                                        void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0 || n < 0 || !d_total || E >= (int64_t(1) << 31)) return PH_ERR_ARG;
  if (n > ph_triangles_total_max_vertices()) {
    record_message("ph_triangles_total_edges: n exceeds the shared-memory bitmap (1638400 vertices)");
    return PH_ERR_ARG;
  }
  Carve c(workspace, workspace_bytes);
  i32* deg = c.take<i32>(n + 1);
  i32* uptr = c.take<i32>(n + 1);
  i32* cursor = c.take<i32>(n + 1);
  i32* uidx = c.take<i32>(std::max<i64>(E, 1));
  void* sws = c.take<char>((i64)scan_workspace_bytes(n));
  int* next = c.take<int>(1);
  if (!deg || !uptr || !cursor || !uidx || !sws || !next) return PH_ERR_ARG;
  ph::zero_async(d_total, sizeof(unsigned long long), s, next, sizeof(int));
  if (n < 3 || E < 3) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  ph::zero_async(deg, sizeof(i32) * (n + 1), s, cursor, sizeof(i32) * (n + 1));
  ph::count_launch();
  ph::launch_pdl(k_upper_deg, dim3(grid_for(E)), dim3(256), 0, s, edge_i, E, deg);
  PH_TRY(scan_exclusive_i32_i32(deg, uptr, n, sws, scan_workspace_bytes(n), s));
  ph::count_launch();
  ph::launch_pdl(k_upper_fill, dim3(grid_for(E)), dim3(256), 0, s, edge_i, edge_j, E, (const i32*)uptr, cursor, uidx);
  const size_t smem = (size_t)((n + 31) / 32) * 4;
  if (smem > 48 * 1024 && ph::allow_dynamic_smem((const void*)k_tri_total<true>) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  const int sms = ph::device_sms();
  const int occ = ph::occupancy((const void*)k_tri_total<true>, SX_NT, smem);
  const int grid = (int)std::max<i64>(1, std::min<i64>(n, (i64)sms * std::max(occ, 1)));
  ph::count_launch();
  ph::launch_pdl(k_tri_total<true>, dim3(grid), dim3(SX_NT), smem, s, (const i32*)uptr, (const i32*)uidx, n, next,
                 d_total, (const i32*)nullptr, (const uint8_t*)nullptr, (unsigned long long*)nullptr);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_triangles_emit(const int32_t* edge_i, const int32_t* edge_j, int64_t E,
                                 const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                                 const int64_t* tri_off, int32_t* tri_m, int32_t* tri_w, int32_t* tri_fa,
                                 int32_t* tri_fb, void* stream) {
  if (E <= 0) return E < 0 ? PH_ERR_ARG : PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_triangles<true>, dim3(warp_grid(E)), dim3(SX_NT), 0, (cudaStream_t)stream, 
      edge_i, edge_j, E, adj_ptr, adj_idx, adj_rank, nullptr, nullptr, tri_off, tri_m, tri_w, tri_fa, tri_fb,
      (const uint8_t*)nullptr, (const i32*)nullptr);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_tets_count_workspace_bytes(int64_t E) {
  return Carve::need((size_t)(E + 1) * 4) + scan_workspace_bytes(E);
}

extern "C" int ph_tets_count(const int64_t* tri_off, const int32_t* tri_w, int64_t E,
                             const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                             const uint8_t* edge_enable, int64_t* tet_off, void* workspace,
                             size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (E < 0) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  i32* qc = c.take<i32>(E + 1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(E));
  if (!qc || !sws) return PH_ERR_ARG;
  if (E > 0) {
    ph::count_launch();
    ph::launch_pdl(k_tets<false>, dim3(warp_grid(E)), dim3(SX_NT), 0, s, nullptr, nullptr, E, tri_off, tri_w, nullptr, nullptr, adj_ptr,
                                                 adj_idx, adj_rank, edge_enable, qc, nullptr, nullptr, nullptr,
                                                 nullptr);
  }
  PH_TRY(scan_exclusive_i32_i64(qc, tet_off, E, sws, scan_workspace_bytes(E), s));
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_tets_emit(const int32_t* edge_i, const int32_t* edge_j, int64_t E, const int64_t* tri_off,
                            const int32_t* tri_w, const int32_t* tri_fa, const int32_t* tri_fb,
                            const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                            const uint8_t* edge_enable, const int64_t* tet_off, int32_t* tet_m,
                            int32_t* tet_faces, int* d_status, void* stream) {
  if (E <= 0) return E < 0 ? PH_ERR_ARG : PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_tets<true>, dim3(warp_grid(E)), dim3(SX_NT), 0, (cudaStream_t)stream, edge_i, edge_j, E, tri_off, tri_w, tri_fa,
                                                                tri_fb, adj_ptr, adj_idx, adj_rank, edge_enable,
                                                                nullptr, tet_off, tet_m, tet_faces, d_status);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" size_t ph_cofacet_csr_workspace_bytes(int64_t S, int32_t k) {
  const i64 H = S * k;
  return Carve::need((size_t)H * 8) + Carve::need((size_t)H * 4) + radix_sort_workspace_bytes(H);
}

extern "C" int ph_cofacet_csr(const int32_t* faces_aos, const int32_t* f0, const int32_t* f1,
                              const int32_t* f2, int32_t k, int64_t S, int64_t n_faces, int32_t row_base,
                              int32_t* cof_off, int32_t* cof_data, void* workspace, size_t workspace_bytes,
                              void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (k < 1 || k > 4 || S < 0 || n_faces < 0) return PH_ERR_ARG;
  if (!faces_aos && (k != 3 || !f0 || !f1 || !f2)) return PH_ERR_ARG;
  const i64 H = S * k;
  if (H >= (int64_t(1) << 31) || (i64)row_base + S >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  if (H == 0) {
    ph::zero_async(cof_off, sizeof(int32_t) * (n_faces + 1), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  u64* keys = c.take<u64>(H);
  u32* vals = c.take<u32>(H);
  void* rws = c.take<char>((i64)radix_sort_workspace_bytes(H));
  if (!keys || !vals || !rws) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_cof_entries, dim3(grid_for(H)), dim3(256), 0, s, faces_aos, f0, f1, f2, k, S, row_base, keys, vals);
  // face indices are below n_faces: sort only the bytes they use (stable, so
  // the simplices of a face stay in ascending order)
  int fb = 1;
  while (fb < 32 && (int64_t(1) << fb) < n_faces) ++fb;
  PH_TRY(radix_sort_pairs(keys, vals, H, 0, std::min(32, ((fb + 7) / 8) * 8), rws, radix_sort_workspace_bytes(H), s));
  ph::count_launch();
  ph::launch_pdl(k_cof_fill, dim3(grid_for(H)), dim3(256), 0, s, keys, vals, H, n_faces, cof_off, cof_data);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int32_t ph_cofacet_rows3_max_row(void) { return RS_BIG; }

extern "C" size_t ph_cofacet_rows3_workspace_bytes(int64_t n_faces) {
  return Carve::need(sizeof(i32) * (size_t)std::max<i64>(n_faces, 1)) * 2 + Carve::need(sizeof(int));
}

extern "C" int ph_cofacet_rows3(const int32_t* f0, const int32_t* f1, const int32_t* f2, int64_t S, int64_t n_faces,
                                int32_t row_base, const int64_t* row_off, int32_t max_row, int32_t* cof_off,
                                int32_t* cof_data, int* d_status, void* workspace, size_t workspace_bytes,
                                void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (S < 0 || n_faces < 0 || !row_off || !cof_off || 3 * S >= (int64_t(1) << 31)) return PH_ERR_ARG;
  if (max_row > RS_BIG) {
    record_message("ph_cofacet_rows3: a row exceeds the in-shared-memory sort; use ph_cofacet_csr");
    return PH_ERR_ARG;
  }
  Carve c(workspace, workspace_bytes);
  i32* cursor = c.take<i32>(std::max<i64>(n_faces, 1));
  i32* big = c.take<i32>(std::max<i64>(n_faces, 1));
  int* nbig = c.take<int>(1);
  if (!cursor || !big || !nbig) return PH_ERR_ARG;
  ph::count_launch();
  ph::launch_pdl(k_off_i64_to_i32, dim3(grid_for(n_faces + 1)), dim3(256), 0, s, row_off, n_faces, cof_off);
  if (S == 0 || n_faces == 0) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  ph::zero_async(cursor, sizeof(i32) * n_faces, s, nbig, sizeof(int));
  ph::count_launch();
  ph::launch_pdl(k_cof_scatter3, dim3(grid_for(S)), dim3(256), 0, s, f0, f1, f2, S, row_base, (const i32*)cof_off,
                 cursor, cof_data, d_status);
  const int gw = (int)std::max<i64>(1, std::min<i64>((n_faces + RS_NT / 32 - 1) / (RS_NT / 32), 148 * 16));
  ph::count_launch();
  ph::launch_pdl(k_cof_sort_rows, dim3(gw), dim3(RS_NT), 0, s, (const i32*)cof_off, n_faces, cof_data, big, nbig);
  ph::count_launch();
  ph::launch_pdl(k_cof_sort_big, dim3(148 * 2), dim3(RS_NT), 0, s, (const i32*)cof_off, cof_data, (const i32*)big,
                 (const int*)nbig, d_status);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

// the largest per-item count given by an exclusive scan: out = max(off[i+1] - off[i])
__global__ void k_max_diff(const i64* __restrict__ off, i64 n, i64* __restrict__ out) {
  ph::pdl_wait();
  ph::pdl_trigger();
  i64 m = 0;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
    m = max(m, off[i + 1] - off[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)m);
}

extern "C" int ph_max_count(const int64_t* off, int64_t n, int64_t* d_out, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !off || !d_out) return PH_ERR_ARG;
  ph::zero_async(d_out, sizeof(int64_t), s);
  if (n > 0) {
    ph::count_launch();
    ph::launch_pdl(k_max_diff, dim3((unsigned)std::max<i64>(1, std::min<i64>((n + 255) / 256, 148 * 8))), dim3(256), 0,
                   s, off, n, d_out);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_cof_max_face(const int32_t* faces_aos, const int32_t* f0, const int32_t* f1,
                               const int32_t* f2, int32_t k, int64_t S, int32_t face_base,
                               const uint8_t* skip, int32_t* cmf, void* stream) {
  if (k < 1 || k > 4 || S < 0) return PH_ERR_ARG;
  if (S == 0) return PH_OK;
  ph::count_launch();
  ph::launch_pdl(k_cmf, dim3(grid_for(S)), dim3(256), 0, (cudaStream_t)stream, faces_aos, f0, f1, f2, k, S, face_base, skip, cmf);
  PH_CHECK_LAUNCH();
  return PH_OK;
}

namespace ph {
size_t cofacet_rows_aos_workspace_bytes(int64_t n_faces) {
  const i64 nf = std::max<i64>(n_faces, 1);
  return Carve::need(sizeof(i32) * (size_t)(nf + 1)) + 2 * Carve::need(sizeof(i32) * (size_t)nf) +
         Carve::need(sizeof(int)) + Carve::need(scan_workspace_bytes(nf));
}

// The cofacet CSR of S simplices with k faces each (AoS, the tetrahedra's four
// triangles) without a sort of the S k entries: rows counted, offsets scanned,
// ranks scattered into their rows, each row sorted in shared memory. Rows must
// hold at most RS_BIG entries (a triangle's tetrahedra number at most the
// cloud's points less three: the caller checks that bound). The rows equal
// ph_cofacet_csr's.
int cofacet_rows_aos(const int32_t* faos, int32_t k, int64_t S, int64_t n_faces, int32_t row_base, int32_t* cof_off,
                     int32_t* cof_data, int* d_status, void* workspace, size_t workspace_bytes, cudaStream_t s) {
  const i64 H = S * k;
  if (k < 1 || S < 0 || n_faces < 0 || H >= (int64_t(1) << 31)) return PH_ERR_ARG;
  Carve c(workspace, workspace_bytes);
  const i64 nf = std::max<i64>(n_faces, 1);
  i32* cnt = c.take<i32>(nf + 1);
  i32* cursor = c.take<i32>(nf);
  i32* big = c.take<i32>(nf);
  int* nbig = c.take<int>(1);
  void* sws = c.take<char>((i64)scan_workspace_bytes(nf));
  if (!cnt || !cursor || !big || !nbig || !sws) return PH_ERR_ARG;
  if (n_faces == 0) {
    ph::zero_async(cof_off, sizeof(i32), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  ph::zero_async(cnt, sizeof(i32) * (size_t)n_faces, s, cursor, sizeof(i32) * (size_t)n_faces);
  ph::zero_async(nbig, sizeof(int), s);
  if (H > 0) {
    ph::count_launch();
    ph::launch_pdl(k_cof_count_aos, dim3(grid_for(H)), dim3(256), 0, s, faos, H, cnt);
  }
  PH_TRY(scan_exclusive_i32_i32(cnt, cof_off, n_faces, sws, scan_workspace_bytes(nf), s));
  if (H == 0) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  ph::count_launch();
  ph::launch_pdl(k_cof_scatter_aos, dim3(grid_for(H)), dim3(256), 0, s, faos, H, (int)k, row_base,
                 (const i32*)cof_off, cursor, cof_data, d_status);
  const int gw = (int)std::max<i64>(1, std::min<i64>((n_faces + RS_NT / 32 - 1) / (RS_NT / 32), 148 * 16));
  ph::count_launch();
  ph::launch_pdl(k_cof_sort_rows, dim3(gw), dim3(RS_NT), 0, s, (const i32*)cof_off, n_faces, cof_data, big, nbig);
  ph::count_launch();
  ph::launch_pdl(k_cof_sort_big, dim3(148 * 2), dim3(RS_NT), 0, s, (const i32*)cof_off, cof_data, (const i32*)big,
                 (const int*)nbig, d_status);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
}  // namespace ph
