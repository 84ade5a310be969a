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
// column as an immutable record and claims the pivot with one atomicMax on the
// pivot's owner word. A smaller column it displaces is taken over by the same
// warp and reduced further. No warp ever waits for another; every loop is
// bounded; running out of pool sets a status code. Apparent columns own their
// pivot from the start and are never displaced (no column processed before an
// apparent column can contain its pivot).
//
// Memory layout. Every column content lives in an immutable record
// [len, rank_0 < rank_1 < ...] in one pool (initial records are copies of the
// cofacet lists; later ones are bump-allocated per warp). The owner word of a
// pivot row is (column + 1) << 33 | record offset, 0 when free, so one
// atomicMax both orders claims by column and publishes the claimer's content:
// a reader needs the owner word and the record, two dependent loads. Claims
// are acquire-release atomics and owner loads are acquire loads, so no full
// fences are needed. The final pivot of each residual column is read from the
// owner table after the kernel.
#include <algorithm>
#include <climits>

#include "prim.cuh"

namespace ph {
namespace {

// Few warps with large shared buffers: the reduction is bound by the latency
// of its dependency chains, not by parallel width, and a working column that
// outgrows its shared buffer falls back to global memory.
constexpr int RD_NT = 128;
constexpr int RD_WARPS = RD_NT / 32;
constexpr int RD_CAP = 6144;   // per-warp shared working-column copies (entries, two of them)
constexpr int RD_CAPB = 2048;  // per-warp shared buffer of the added column
constexpr int RD_WSTRIDE = 2 * RD_CAP + RD_CAPB;
constexpr size_t RD_SMEM = (size_t)RD_WARPS * RD_WSTRIDE * sizeof(int32_t);
constexpr unsigned FULL = 0xffffffffu;
constexpr int RD_FETCH = 8;  // columns a warp takes from the descending sweep at a time
constexpr int OW_SHIFT = 33;
constexpr u64 OW_OFF = (1ull << OW_SHIFT) - 1;

struct RedCtl {
  int nres;
  int next;
  int abort;
  int pad;
  unsigned long long pool_top;
  unsigned long long merges;
  unsigned long long takeovers;
};

__device__ __forceinline__ u64 owner_word(i32 c, u64 off) { return ((u64)(c + 1) << OW_SHIFT) | off; }
__device__ __forceinline__ i32 owner_col(u64 w) { return (i32)(w >> OW_SHIFT) - 1; }

__device__ __forceinline__ u64 ld_acquire(const u64* p) {
  u64 v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ u64 atom_max_acq_rel(u64* p, u64 v) {
  u64 old;
  asm volatile("atom.acq_rel.gpu.global.max.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

// Classifies columns; gives every non-empty column an initial record; apparent
// columns own their pivot; residual columns (state 2) are left for the
// reducer. Record space is taken with one atomic per warp.
__global__ void k_classify(const i32* __restrict__ off, const i32* __restrict__ cof, i64 K, i32 col_base,
                           i32 row_base, const uint8_t* __restrict__ skip, const i32* __restrict__ cmf,
                           i32* __restrict__ state, i32* __restrict__ piv, u64* __restrict__ owner,
                           u64* __restrict__ rec, i32* __restrict__ pool, i64 pool_cap, RedCtl* ctl, int* status) {
  ph::pdl_wait();
  ph::pdl_trigger();
  const int lane = threadIdx.x & 31;
  const i64 stride = (i64)gridDim.x * blockDim.x;
  for (i64 c0 = (i64)blockIdx.x * blockDim.x + (threadIdx.x & ~31); c0 < K; c0 += stride) {
    const i64 c = c0 + lane;
    int len = 0;
    bool skipped = false, resid_col = false;
    i32 o0 = 0, t = 0;
    if (c < K) {
      o0 = off[c];
      len = off[c + 1] - o0;
      skipped = skip && skip[c];
      if (skipped) {
        state[c] = 0;
        piv[c] = -1;
      } else if (len == 0) {
        state[c] = 3;
        piv[c] = -1;
      } else {
        t = cof[o0];
        resid_col = cmf[t - row_base] != col_base + (i32)c;
      }
    }
    const bool has = c < K && !skipped && len > 0;
    // warp prefix of record sizes
    int need = has ? len + 1 : 0, incl = need;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total) base = atomicAdd(&ctl->pool_top, (unsigned long long)total);
    base = __shfl_sync(FULL, base, 31);
    const u32 rm = __ballot_sync(FULL, resid_col);
    if (lane == 0 && rm) atomicAdd(&ctl->nres, __popc(rm));
    if (!has) continue;
    const unsigned long long at = base + (unsigned long long)(incl - need);
    if (base + (unsigned long long)total > (unsigned long long)pool_cap) {
      set_status(status, PH_ERR_POOL);
      atomicExch(&ctl->abort, 1);
      state[c] = 3;
      piv[c] = -1;
      continue;
    }
    pool[at] = len;
    for (int i = 0; i < len; ++i) pool[at + 1 + i] = cof[o0 + i];
    if (!resid_col) {
      state[c] = 1;
      piv[c] = t;
      owner[t - row_base] = owner_word((i32)c, at);
    } else {
      state[c] = 2;
      rec[c] = at;
    }
  }
}

// Loads that must see data written by other SMs during this kernel go to L2.
template <bool G>
__device__ __forceinline__ i32 ld(const i32* p) {
  if (G) return __ldcg(p);
  return *p;
}

// out = L xor S for L (<= 32 MR entries, in registers) and S (ns <= 32, one
// per lane in sv). An element's output position is its rank in its own list
// plus its rank in the other list, less twice the common values below it;
// common values are dropped. The ranks of L's entries in S come from ns
// broadcasts of S (independent shuffles, so their latencies overlap). L being
// sorted, those ranks are non-decreasing, and the S entries that fall between
// L[i-1] and L[i] are exactly S[rank(L[i-1]) ..< rank(L[i])] (past a common
// value): the lane holding L[i] writes them, knowing their rank in L (i)
// without any search. S entries above all of L are written by their own lanes.
template <bool G, int MR>
__device__ int warp_xor_tiny(const i32* L, int nl, i32 sv, int ns, i32* out) {
  const int lane = threadIdx.x & 31;
  const u32 lt = lanemask_lt();
  i32 lr[MR];
  int rs[MR];
  bool eq[MR], valid[MR];
#pragma unroll
  for (int m = 0; m < MR; ++m) {
    valid[m] = lane + 32 * m < nl;
    lr[m] = valid[m] ? ld<G>(L + lane + 32 * m) : INT_MAX;
    rs[m] = 0;
    eq[m] = false;
  }
  for (int j0 = 0; j0 < ns; j0 += 8) {  // eight broadcasts in flight at a time
    i32 s[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) s[q] = __shfl_sync(FULL, sv, (j0 + q) & 31);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (j0 + q < ns) {
#pragma unroll
        for (int m = 0; m < MR; ++m) {
          rs[m] += s[q] < lr[m];
          eq[m] |= s[q] == lr[m];
        }
      }
  }
  u32 dm[MR];
  int before[MR];
  int dtot = 0;
#pragma unroll
  for (int m = 0; m < MR; ++m) {
    dm[m] = __ballot_sync(FULL, eq[m] && valid[m]);
    before[m] = dtot;
    dtot += __popc(dm[m]);
  }
  // L's entries
  int lo[MR], span = 0;
#pragma unroll
  for (int m = 0; m < MR; ++m) {
    const int i = lane + 32 * m;
    const int d = before[m] + __popc(dm[m] & lt);
    if (valid[m] && !eq[m]) out[i + rs[m] - 2 * d] = lr[m];
    // first S index after L[i-1] (past it when they are equal)
    int prev = __shfl_up_sync(FULL, rs[m] + (int)eq[m], 1);
    if (m > 0) {
      const int last = __shfl_sync(FULL, rs[m - 1] + (int)eq[m - 1], 31);
      if (lane == 0) prev = last;
    } else if (lane == 0) {
      prev = 0;
    }
    lo[m] = prev;
    if (valid[m]) span = max(span, rs[m] - lo[m]);
  }
  span = __reduce_max_sync(FULL, span);
  // S entries between L[i-1] and L[i], written by the lane holding L[i]
  for (int t = 0; t < span; ++t) {
#pragma unroll
    for (int m = 0; m < MR; ++m) {
      const int j = lo[m] + t;
      const i32 v = __shfl_sync(FULL, sv, j & 31);
      if (valid[m] && j < rs[m]) out[j + lane + 32 * m - 2 * (before[m] + __popc(dm[m] & lt))] = v;
    }
  }
  // S entries above all of L
  int lo_end = 0;
  if (nl > 0) {
    const int ml = (nl - 1) >> 5, ll = (nl - 1) & 31;
#pragma unroll
    for (int m = 0; m < MR; ++m)
      if (m == ml) lo_end = __shfl_sync(FULL, rs[m] + (int)eq[m], ll);
  }
  if (lane < ns && lane >= lo_end) out[lane + nl - 2 * dtot] = sv;
  return nl + ns - 2 * dtot;
}

// out = L xor S for a sorted list L of distinct ranks and a sorted list S of
// at most 32 distinct ranks held one per lane (sv; INT_MAX beyond ns) -- the
// common shape: a long working column and a short added one. Lane j finds S_j
// in L by binary search; S_j lands at pos_j + j - 2 D_j (D_j = duplicates
// among S_0..S_{j-1}), and L splits into ns + 1 segments between the insertion
// points, each moved by one constant shift: the warp copies long segments one
// after another, short ones 32 elements at a time. Returns the (warp-uniform)
// output length.
template <bool G>
__device__ int warp_xor_small(const i32* L, int nl, i32 sv, int ns, i32* out) {
  if (nl <= 32) return warp_xor_tiny<G, 1>(L, nl, sv, ns, out);
  if (nl <= 64) return warp_xor_tiny<G, 2>(L, nl, sv, ns, out);
  if (nl <= 128) return warp_xor_tiny<G, 4>(L, nl, sv, ns, out);
  if (nl <= 256) return warp_xor_tiny<G, 8>(L, nl, sv, ns, out);
  const int lane = threadIdx.x & 31;
  const u32 lt = lanemask_lt();
  const bool act = lane < ns;
  int pos = nl;
  if (act) {
    int lo = 0, hi = nl;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ld<G>(L + mid) < sv) lo = mid + 1;
      else hi = mid;
    }
    pos = lo;
  }
  const bool dup = act && pos < nl && ld<G>(L + pos) == sv;
  const u32 dm = __ballot_sync(FULL, dup);
  if (act && !dup) out[pos + lane - 2 * __popc(dm & lt)] = sv;
  if (nl >= 64 * (ns + 1)) {
    // long segments: the warp copies segment k = 0..ns in turn, moved by k - 2 D_k
    const int pprev = __shfl_up_sync(FULL, pos, 1);
    const int start = lane == 0 ? 0 : pprev + (int)((dm >> (lane - 1)) & 1u);
    for (int k = 0; k <= ns && k < 32; ++k) {
      const int a = __shfl_sync(FULL, start, k);
      const int b = k == ns ? nl : __shfl_sync(FULL, pos, k);
      const int sh = k - 2 * __popc(dm & ((1u << k) - 1u));
      for (int i = a + lane; i < b; i += 32) out[i + sh] = ld<G>(L + i);
    }
    if (ns == 32) {  // segment 32 (after the last insertion point)
      const int a = __shfl_sync(FULL, pos, 31) + (int)(dm >> 31), sh = 32 - 2 * __popc(dm);
      for (int i = a + lane; i < nl; i += 32) out[i + sh] = ld<G>(L + i);
    }
  } else {
    // short segments: 32 elements of L at a time; c = #{j : pos_j <= i} by
    // broadcast shuffles of the insertion points, L[i] deleted when S_{c-1} is
    // its twin, else moved by c - 2 D_c
    for (int i0 = 0; i0 < nl; i0 += 32) {
      const int i = i0 + lane;
      int c = 0;
      for (int j = 0; j < ns; ++j) c += __shfl_sync(FULL, pos, j) <= i;
      const int plast = __shfl_sync(FULL, pos, (c + 31) & 31);
      const u32 below = c >= 32 ? FULL : ((1u << c) - 1u);
      const bool deleted = c > 0 && ((dm >> (c - 1)) & 1u) && plast == i;
      if (i < nl && !deleted) out[i + c - 2 * __popc(dm & below)] = ld<G>(L + i);
    }
  }
  return nl + ns - 2 * __popc(dm);
}

// out = A xor B for sorted lists of distinct ranks, both longer than 32, by
// merge path over 128 segments of the merged sequence (ties: A first): lane l
// merges segments 4l .. 4l + 3 as four interleaved chains (independent loads
// in flight), counting survivors in a first pass and writing them after a
// scan. An element is dropped when its twin is in the other list; the twin of
// A[i] can only be B[ib] and the twin of B[j] only A[ia - 1] at the merge
// position, whichever segment they fall in. The loop is branch-free so that
// lanes do not diverge.
template <bool AG, bool BG>
__device__ int warp_xor_merge(const i32* A, int na, const i32* B, int nb, i32* out) {
  constexpr int CH = 4;
  const int lane = threadIdx.x & 31;
  const int total = na + nb;
  const int per = (total + 32 * CH - 1) / (32 * CH);
  int ia0[CH], ib0[CH], d1[CH];
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    const int d0 = min((lane * CH + c) * per, total);
    d1[c] = min(d0 + per, total);
    int lo = max(0, d0 - nb), hi = min(d0, na);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ld<AG>(A + mid) <= ld<BG>(B + d0 - 1 - mid)) lo = mid + 1;
      else hi = mid;
    }
    ia0[c] = lo;
    ib0[c] = d0 - lo;
  }
  int cnt[CH] = {0, 0, 0, 0};
  int total_out = 0;
  for (int pass = 0; pass < 2; ++pass) {
    int ia[CH], ib[CH], pos[CH], d[CH];
    i32 a[CH], b[CH], pa[CH];
    int lane_base = 0;
    if (pass == 1) {
      const int mine = cnt[0] + cnt[1] + cnt[2] + cnt[3];
      int incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      lane_base = incl - mine;
      total_out = __shfl_sync(FULL, incl, 31);
    }
    int run = lane_base;
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      ia[c] = ia0[c];
      ib[c] = ib0[c];
      d[c] = ia0[c] + ib0[c];
      a[c] = ia[c] < na ? ld<AG>(A + ia[c]) : INT_MAX;
      b[c] = ib[c] < nb ? ld<BG>(B + ib[c]) : INT_MAX;
      pa[c] = ia[c] > 0 ? ld<AG>(A + ia[c] - 1) : -1;
      pos[c] = run;
      run += cnt[c];
      if (pass == 0) cnt[c] = 0;
    }
    for (int step = 0; step < per; ++step) {
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (d[c] >= d1[c]) continue;
        const bool ta = ib[c] >= nb || (ia[c] < na && a[c] <= b[c]);
        const i32 x = ta ? a[c] : b[c];
        const bool keep = ta ? (b[c] != a[c]) : (pa[c] != b[c]);
        if (pass == 1 && keep) out[pos[c]] = x;
        pos[c] += keep;
        if (pass == 0) cnt[c] += keep;
        pa[c] = ta ? a[c] : pa[c];
        ia[c] += ta;
        ib[c] += !ta;
        ++d[c];
        const i32 an = ld<AG>(A + min(ia[c], na - 1)), bn = ld<BG>(B + min(ib[c], nb - 1));
        a[c] = ia[c] < na ? an : INT_MAX;
        b[c] = ib[c] < nb ? bn : INT_MAX;
      }
    }
  }
  return total_out;
}

__device__ __forceinline__ int symdiff(const i32* A, bool ag, int na, const i32* B, bool bg, int nb, i32* out) {
  const int lane = threadIdx.x & 31;
  if (nb <= 32) {
    const i32 sv = lane < nb ? (bg ? __ldcg(B + lane) : B[lane]) : INT_MAX;
    return ag ? warp_xor_small<true>(A, na, sv, nb, out) : warp_xor_small<false>(A, na, sv, nb, out);
  }
  if (na <= 32) {
    const i32 sv = lane < na ? (ag ? __ldcg(A + lane) : A[lane]) : INT_MAX;
    return bg ? warp_xor_small<true>(B, nb, sv, na, out) : warp_xor_small<false>(B, nb, sv, na, out);
  }
  if (ag) return bg ? warp_xor_merge<true, true>(A, na, B, nb, out) : warp_xor_merge<true, false>(A, na, B, nb, out);
  return bg ? warp_xor_merge<false, true>(A, na, B, nb, out) : warp_xor_merge<false, false>(A, na, B, nb, out);
}

// Per-warp bump allocation from pool chunks (lane 0 holds the chunk); the
// offset is broadcast to the warp, ~0 when the pool is exhausted.
struct PoolChunk {
  unsigned long long pos = 0, end = 0;
};

__device__ __forceinline__ unsigned long long pool_alloc(PoolChunk& ch, RedCtl* ctl, i64 cap, int n, int chunk,
                                                         int* status) {
  unsigned long long at = 0;
  if ((threadIdx.x & 31) == 0) {
    if (ch.pos + (unsigned long long)n <= ch.end) {
      at = ch.pos;
      ch.pos += n;
    } else {
      const int take = n > chunk / 2 ? n : chunk;
      at = atomicAdd(&ctl->pool_top, (unsigned long long)take);
      if (at + (unsigned long long)take > (unsigned long long)cap) {
        set_status(status, PH_ERR_POOL);
        atomicExch(&ctl->abort, 1);
        at = ~0ull;
      } else if (take > n) {
        ch.pos = at + n;
        ch.end = at + take;
      }
    }
  }
  return __shfl_sync(FULL, at, 0);
}

// ---- dense working columns ---------------------------------------------------------
// A working column can be a bitmap over the row range, private to its warp
// (cleared on first use and after each column): adding a column flips its
// bits, the next pivot is the first set bit at or after the current one (the
// added column's entries are all >= the pivot it cancels), and the sorted
// record is produced only when the column claims a pivot. Cost per addition
// is the added column's length, not the working column's. When the row range
// fits one of the warp's shared buffers (up to 32 * RD_CAP rows) every
// working column is such a bitmap in shared memory; otherwise only a column
// that outgrows its shared buffer becomes one, in a global slot per warp.
//
// A global bitmap spans the whole row range (millions of rows for dense
// complexes), while a column's entries are a few thousand at most: scanning
// it word by word for the next pivot, the record or the clear would cost the
// range, not the column. Global bitmaps therefore carry a summary in the
// warp's shared memory: bit b of summary word s is set when data words
// [32 (32 s + b), 32 (32 s + b) + 32) (1024 rows, one warp-wide load) may hold
// set bits. Flips set summary bits; scans visit only the blocks whose bits
// are set and drop the bits of blocks found empty; clearing a column zeroes
// only its blocks.
constexpr int RD_SUM_WORDS = RD_CAPB;  // summary words (the added-column buffer, idle while the column is a bitmap)

struct DenseCol {
  u32* bits = nullptr;  // this warp's bitmap
  u32* sum = nullptr;   // summary of a global bitmap (shared memory), null for a shared bitmap
  i32 rb = 0;           // rank of the bitmap's bit 0 (word-aligned, at or below the column's first pivot)
  i64 lo = 0, hi = -1;  // touched word range
  i32 piv = -1;         // lowest set bit (global rank)
  bool sm = false;      // bits are in this warp's shared memory
};

// shared-memory forms of the bitmap accesses (explicit state space: the
// bitmap pointer is generic, and generic atomics and loads take a slower path)
__device__ __forceinline__ u32 sm_ld32(const u32* p) {
  u32 v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"((u32)__cvta_generic_to_shared(p)) : "memory");
  return v;
}
__device__ __forceinline__ u32 sm_xor32(u32* p, u32 x) {
  u32 old;
  asm volatile("atom.shared.xor.b32 %0, [%1], %2;" : "=r"(old) : "r"((u32)__cvta_generic_to_shared(p)), "r"(x)
               : "memory");
  return old;
}
__device__ __forceinline__ void sm_red_xor32(u32* p, u32 x) {
  asm volatile("red.shared.xor.b32 [%0], %1;" ::"r"((u32)__cvta_generic_to_shared(p)), "r"(x) : "memory");
}
__device__ __forceinline__ void sm_red_or32(u32* p, u32 x) {
  asm volatile("red.shared.or.b32 [%0], %1;" ::"r"((u32)__cvta_generic_to_shared(p)), "r"(x) : "memory");
}
__device__ __forceinline__ void sm_red_and32(u32* p, u32 x) {
  asm volatile("red.shared.and.b32 [%0], %1;" ::"r"((u32)__cvta_generic_to_shared(p)), "r"(x) : "memory");
}
__device__ __forceinline__ void gl_red_xor32(u32* p, u32 x) {
  asm volatile("red.relaxed.gpu.global.xor.b32 [%0], %1;" ::"l"(p), "r"(x) : "memory");
}

__device__ __forceinline__ void sm_st32(u32* p, u32 v) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"((u32)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}

__device__ __forceinline__ u32 dense_word(const DenseCol& D, i64 w) { return D.sm ? sm_ld32(D.bits + w) : __ldcg(D.bits + w); }
__device__ __forceinline__ u32 dense_xor(const DenseCol& D, i64 w, u32 b) {
  return D.sm ? sm_xor32(D.bits + w, b) : atomicXor(D.bits + w, b);
}

// flips the sorted entries src[0..len) (global ranks); returns the change in
// the number of set bits (warp-uniform) and widens the touched range
// flips the sorted entries held one per lane (lanes < len <= 32); the set-bit
// count is not tracked here (the flips need not return their old words): a
// vanished column shows as no set bit at the pivot scan, and the count of a
// column is taken when it is published
__device__ void dense_flip_regs(DenseCol& D, i32 v, int len, i32 row_base) {
  const int lane = threadIdx.x & 31;
  if (lane < len) {
    const i32 e = v - row_base;
    const u32 b = 1u << (e & 31);
    if (D.sm) {
      sm_red_xor32(D.bits + (e >> 5), b);
    } else {
      gl_red_xor32(D.bits + (e >> 5), b);
      if (D.sum) sm_red_or32(D.sum + (e >> 15), 1u << ((e >> 10) & 31));
    }
  }
  if (!D.sm) __threadfence_block();
  const i32 first = __shfl_sync(FULL, v, 0), last = __shfl_sync(FULL, v, (len - 1) & 31);
  if (len > 0) {
    const i64 w0 = (i64)((first - row_base) >> 5), w1 = (i64)((last - row_base) >> 5);
    D.lo = D.hi < D.lo ? w0 : min(D.lo, w0);
    D.hi = max(D.hi, w1);
  }
  __syncwarp();
}

// Calls f(block) (warp-uniform) for every block of 32 data words in [b0, b1]
// whose summary bit is set, in ascending order; f returns false to stop.
template <typename F>
__device__ __forceinline__ void for_each_block(const DenseCol& D, i64 b0, i64 b1, F&& f) {
  const int lane = threadIdx.x & 31;
  for (i64 s0 = (b0 >> 5); s0 <= (b1 >> 5); s0 += 32) {
    const i64 sw = s0 + lane;
    u32 m = sw <= (b1 >> 5) ? sm_ld32(D.sum + sw) : 0u;
    if (sw == (b0 >> 5)) m &= ~0u << (b0 & 31);
    if (sw == (b1 >> 5) && (b1 & 31) != 31) m &= (2u << (b1 & 31)) - 1u;
    u32 lanes = __ballot_sync(FULL, m != 0);
    while (lanes) {
      const int l = __ffs(lanes) - 1;
      lanes &= lanes - 1;
      u32 bits = __shfl_sync(FULL, m, l);
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        if (!f(((s0 + l) << 5) + b)) return;
      }
    }
  }
}

// Lane-parallel walk over the blocks of [b0, b1] whose summary bits are set:
// one summary word (up to 32 blocks) per step, lane l taking the step's l-th
// block, so a lane reads a whole block (128 bytes, eight 16-byte loads in
// flight) and a step costs one memory round trip however many blocks it
// covers. g(block, active) is called by every lane (warp-uniform control
// flow); active is false on lanes without a block this step.
template <typename G>
__device__ __forceinline__ void for_each_block_lanes(const DenseCol& D, i64 b0, i64 b1, G&& g) {
  const int lane = threadIdx.x & 31;
  for (i64 sw = (b0 >> 5); sw <= (b1 >> 5); ++sw) {
    u32 m = sm_ld32(D.sum + sw);
    if (sw == (b0 >> 5)) m &= ~0u << (b0 & 31);
    if (sw == (b1 >> 5) && (b1 & 31) != 31) m &= (2u << (b1 & 31)) - 1u;
    if (!m) continue;
    const bool active = lane < __popc(m);
    const i64 blk = active ? (sw << 5) + (i64)__fns(m, 0, lane + 1) : 0;
    g(blk, active);
  }
}

// the 32 words of block b, those outside [wlo, whi] as zero
__device__ __forceinline__ void load_block(const DenseCol& D, i64 b, i64 wlo, i64 whi, u32 (&v)[32]) {
  const uint4* p = reinterpret_cast<const uint4*>(D.bits + (b << 5));
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const uint4 x = __ldcg(p + q);
    v[4 * q + 0] = x.x;
    v[4 * q + 1] = x.y;
    v[4 * q + 2] = x.z;
    v[4 * q + 3] = x.w;
  }
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const i64 w = (b << 5) + k;
    if (w < wlo || w > whi) v[k] = 0u;
  }
}

// set bits of the bitmap (all at or after the pivot's word)
__device__ int dense_count(const DenseCol& D, i32 row_base) {
  const int lane = threadIdx.x & 31;
  int c = 0;
  const i64 w0 = (i64)((D.piv - row_base) >> 5);
  if (D.sum) {
    for_each_block_lanes(D, w0 >> 5, D.hi >> 5, [&](i64 b, bool active) {
      if (!active) return;
      u32 v[32];
      load_block(D, b, w0, D.hi, v);
#pragma unroll
      for (int k = 0; k < 32; ++k) c += __popc(v[k]);
    });
    return __reduce_add_sync(FULL, c);
  }
  for (i64 w = w0 + lane; w <= D.hi; w += 32) c += __popc(dense_word(D, w));
  return __reduce_add_sync(FULL, c);
}

// one entry's flip: the bitmap bit, and the summary bit of its block
__device__ __forceinline__ void dense_flip1(const DenseCol& D, i32 e) {
  const u32 b = 1u << (e & 31);
  if (D.sm) {
    sm_red_xor32(D.bits + (e >> 5), b);
  } else {
    gl_red_xor32(D.bits + (e >> 5), b);
    if (D.sum) sm_red_or32(D.sum + (e >> 15), 1u << ((e >> 10) & 31));
  }
}

// flips the sorted entries src[0..len) (global ranks) and widens the touched
// range. Flips are fire-and-forget reductions (nothing waits for the old
// words; the set-bit count is taken when the column is published), with eight
// source loads per lane in flight: an added column can hold 10^5 entries.
__device__ void dense_flip(DenseCol& D, const i32* src, bool srcg, int len, i32 row_base) {
  const int lane = threadIdx.x & 31;
  int i = lane;
  for (; i + 224 < len; i += 256) {
    i32 e[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) e[q] = (srcg ? __ldcg(src + i + 32 * q) : src[i + 32 * q]) - row_base;
#pragma unroll
    for (int q = 0; q < 8; ++q) dense_flip1(D, e[q]);
  }
  for (; i < len; i += 32) dense_flip1(D, (srcg ? __ldcg(src + i) : src[i]) - row_base);
  if (len > 0) {
    const i64 w0 = (i64)(((srcg ? __ldcg(src) : src[0]) - row_base) >> 5);
    const i64 w1 = (i64)(((srcg ? __ldcg(src + len - 1) : src[len - 1]) - row_base) >> 5);
    D.lo = D.hi < D.lo ? w0 : min(D.lo, w0);
    D.hi = max(D.hi, w1);
  }
  // the flips are visible to the warp's later loads of the bitmap
  if (!D.sm) __threadfence_block();
  __syncwarp();
}

// first set bit at or after word `from` (global rank), -1 if none
__device__ i32 dense_first(const DenseCol& D, i64 from, i32 row_base) {
  const int lane = threadIdx.x & 31;
  if (D.sum) {
    i32 found = -1;
    for_each_block(D, from >> 5, D.hi >> 5, [&](i64 b) {
      const i64 w = (b << 5) + lane;
      const u32 v = (w >= from && w <= D.hi) ? __ldcg(D.bits + w) : 0u;
      const u32 m = __ballot_sync(FULL, v != 0);
      if (m) {
        const int f = __ffs(m) - 1;
        const u32 vw = __shfl_sync(FULL, v, f);
        found = (i32)((((b << 5) + f) << 5) + (__ffs(vw) - 1)) + row_base;
        return false;
      }
      // an empty block (every bit it held was flipped away): drop its summary
      // bit, unless part of it lies before `from` (those words were not read)
      if ((b << 5) >= from && lane == 0) sm_red_and32(D.sum + (b >> 5), ~(1u << (b & 31)));
      __syncwarp();
      return true;
    });
    return found;
  }
  for (i64 w0 = from; w0 <= D.hi; w0 += 32) {
    const i64 w = w0 + lane;
    const u32 v = w <= D.hi ? dense_word(D, w) : 0u;
    const u32 m = __ballot_sync(FULL, v != 0);
    if (m) {
      const int f = __ffs(m) - 1;
      const u32 vw = __shfl_sync(FULL, v, f);
      return (i32)(((w0 + f) << 5) + (__ffs(vw) - 1)) + row_base;
    }
  }
  return -1;
}

// the set bits from the pivot's word on, ascending, into out[0..k)
__device__ void dense_to_list(const DenseCol& D, i32 row_base, i32* out) {
  const int lane = threadIdx.x & 31;
  int pos = 0;
  const i64 wp = (i64)((D.piv - row_base) >> 5);
  if (D.sum) {
    for_each_block_lanes(D, wp >> 5, D.hi >> 5, [&](i64 b, bool active) {
      u32 v[32];
      int c = 0;
      if (active) {
        load_block(D, b, wp, D.hi, v);
#pragma unroll
        for (int k = 0; k < 32; ++k) c += __popc(v[k]);
      }
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += t;
      }
      if (active) {  // the lane's block is the lane-th of the step in ascending order
        int at = pos + incl - c;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          u32 x = v[k];
          while (x) {
            out[at++] = (i32)((((b << 5) + k) << 5) + (__ffs(x) - 1)) + row_base;
            x &= x - 1;
          }
        }
      }
      pos += __shfl_sync(FULL, incl, 31);
    });
    __syncwarp();
    return;
  }
  for (i64 w0 = wp; w0 <= D.hi; w0 += 32) {
    const i64 w = w0 + lane;
    u32 v = w <= D.hi ? dense_word(D, w) : 0u;
    const int c = __popc(v);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    int q = pos + incl - c;
    while (v) {
      out[q++] = (i32)((w << 5) + (__ffs(v) - 1)) + row_base;
      v &= v - 1;
    }
    pos += __shfl_sync(FULL, incl, 31);
  }
  __syncwarp();
}

// zeroes the summary words of blocks [b0, b1]
__device__ void dense_sum_zero(DenseCol& D, i64 b0, i64 b1) {
  const int lane = threadIdx.x & 31;
  for (i64 sw = (b0 >> 5) + lane; sw <= (b1 >> 5); sw += 32) sm_st32(D.sum + sw, 0u);
  __syncwarp();
}

__device__ void dense_clear(DenseCol& D, i64 lo, i64 hi) {
  const int lane = threadIdx.x & 31;
  if (D.sum && hi >= lo) {  // only the blocks that may hold set bits
    for_each_block_lanes(D, lo >> 5, hi >> 5, [&](i64 b, bool active) {
      if (!active) return;
      uint4* p = reinterpret_cast<uint4*>(D.bits + (b << 5));
#pragma unroll
      for (int q = 0; q < 8; ++q) __stcg(p + q, make_uint4(0u, 0u, 0u, 0u));
    });
    __syncwarp();
    dense_sum_zero(D, lo >> 5, hi >> 5);
    D.lo = 0;
    D.hi = -1;
    D.piv = -1;
    return;
  }
  if (D.sm)
    for (i64 w = lo + lane; w <= hi; w += 32) sm_st32(D.bits + w, 0u);
  else
    for (i64 w = lo + lane; w <= hi; w += 32) __stcg(D.bits + w, 0u);
  __syncwarp();
  D.lo = 0;
  D.hi = -1;
  D.piv = -1;
}

// Residual columns are taken in descending order (the serial algorithm's
// order), RD_FETCH at a time per warp, so that a column mostly meets final
// versions of the larger columns it adds and is rarely displaced.
__global__ void __launch_bounds__(RD_NT, 1) k_reduce(i32 row_base, i64 K, const i32* __restrict__ state,
                                                 const u64* __restrict__ rec, u64* owner, i32* pool, i64 pool_cap,
                                                 int chunk, RedCtl* ctl, int* status, int max_steps,
                                                 u32* dense_bits, i64 dense_words, int sm_words) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ i32 rd_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  i32* const sW0 = rd_smem + (size_t)w * RD_WSTRIDE;  // working copies at sW0 and sW0 + RD_CAP
  i32* const sBw = sW0 + 2 * RD_CAP;
  volatile int* vabort = &ctl->abort;
  PoolChunk chunk_state;
  unsigned long long n_merges = 0, n_takeovers = 0;
  DenseCol D;
  bool dense_ready = false;  // this warp's slot has been cleared once
  // shared bitmap (in the second working buffer) when the rows fit, else the global slot
  const bool dense_sm = sm_words > 0;
  const bool dense_ok = dense_sm || dense_words > 0;
  const i64 dwords = dense_sm ? (i64)sm_words : dense_words;
  if (dense_sm) {
    D.bits = reinterpret_cast<u32*>(sW0 + RD_CAP);
    D.sm = true;
  } else if (dense_ok) {
    D.bits = dense_bits + (size_t)(blockIdx.x * RD_WARPS + w) * (size_t)dense_words;
    // the summary needs one bit per 32 data words; a slot's word count is
    // bounded by the 1 GiB of slots, far below RD_SUM_WORDS * 1024 words
    if ((dense_words + 1023) / 1024 <= RD_SUM_WORDS) D.sum = reinterpret_cast<u32*>(sBw);
  }
  const i64 sum_blocks = (dwords + 31) / 32;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&ctl->next, RD_FETCH);
    base = __shfl_sync(FULL, base, 0);
    if ((i64)base >= K || *vabort) break;
    const i64 cand = K - 1 - base - lane;
    u32 todo = __ballot_sync(FULL, lane < RD_FETCH && cand >= 0 && state[cand] == 2);
    while (todo && !*vabort) {
    const int l = __ffs(todo) - 1;
    todo &= todo - 1;
    i32 c = (i32)(K - 1 - base - l);
    // working column: shared buffer (sW0 + cur * RD_CAP), a pool record when too
    // long, or the bitmap D
    int cur = 0;
    int k = 0;  // entries of W; for the bitmap only zero/nonzero until it is published
    const i32* W = nullptr;
    bool wg = false;      // W is in global memory
    bool published = false;
    u64 wrec = 0;         // record offset of W when published
    bool dense = false;   // W is the bitmap D
    auto enter_dense = [&](const i32* src, bool srcg, int len) {
      // the summary shares its buffer with the list form's added-column copy:
      // zero it whenever a column becomes a bitmap
      if (D.sum) dense_sum_zero(D, 0, sum_blocks - 1);
      if (!dense_ready) {
        u32* keep = D.sum;
        D.sum = nullptr;  // the first clear covers the whole slot (its content is unknown)
        dense_clear(D, 0, dwords - 1);
        D.sum = keep;
        dense_ready = true;
      }
      D.piv = len > 0 ? (srcg ? __ldcg(src) : src[0]) : -1;
      // the column's entries stay within [first pivot, first pivot + span):
      // the bitmap window starts at the first pivot's word
      D.rb = len > 0 ? row_base + (((D.piv - row_base) >> 5) << 5) : row_base;
      dense_flip(D, src, srcg, len, D.rb);
      if (D.sm) {  // a shared bitmap is read and cleared whole: no touched range to track
        D.lo = 0;
        D.hi = dwords - 1;
      }
      dense = true;
    };
    auto leave_dense = [&]() {
      if (dense) dense_clear(D, D.lo, D.hi);
      dense = false;
    };
    auto load_record = [&](u64 at) {
      const i32* src = pool + at + 1;
      k = __ldcg(pool + at);
      if (dense_sm || (k > RD_CAP && dense_ok)) {
        enter_dense(src, true, k);
      } else if (k <= RD_CAP) {
        for (int i = lane; i < k; i += 32) (sW0 + cur * RD_CAP)[i] = __ldcg(src + i);
        __syncwarp();
        W = (sW0 + cur * RD_CAP);
        wg = false;
      } else {
        W = src;
        wg = true;
      }
      wrec = at;
      published = true;
    };
    load_record(rec[c]);
    // After a takeover the working column still holds the content of the
    // column that just claimed the pivot, and the displaced column must add
    // exactly that content: the step adds the displaced record to it instead
    // of loading the displaced record and then re-reading the owner word and
    // the record just published (two fewer dependent L2 round trips on the
    // takeover chains that form the critical path).
    u64 pending = 0;
    for (int step = 0;; ++step) {
      // another warp's abort (pool exhausted) is checked every 64 steps: the
      // flag is an L2 round trip, as long as a whole step of a short column
      if (dense && (step & 63) == 63 && *vabort) break;
      if (step >= max_steps) {
        if (lane == 0) set_status(status, PH_ERR_ITER_LIMIT);
        atomicExch(&ctl->abort, 1);
        break;
      }
      if (k == 0) break;  // the column vanished: it owns nothing
      const bool take = pending != 0;
      // The chain of additions of a shared-bitmap column, in a loop of its own:
      // while its pivot's owner is a larger column, add that column's record
      // (one owner-word and one record-head round trip), then find the new
      // pivot from the old one's word on. Long columns spend their whole
      // reduction here, and this loop's few branches and registers make a
      // step about 1.5x shorter than one of the general loop below, which
      // takes over at the first pivot the column must claim (its owner word
      // already loaded).
      u64 ow_known = 0;
      bool have_ow = false, aborted = false;
      if (dense && D.sm && !take) {
        for (;;) {
          const i32 pf = D.piv;
          const u64 ow_f = ld_acquire(owner + (pf - row_base));
          if (owner_col(ow_f) <= c) {
            ow_known = ow_f;
            have_ow = true;
            break;
          }
          const u64 at_f = ow_f & OW_OFF;
          const i32 head = (at_f + lane < (u64)pool_cap) ? __ldcg(pool + at_f + lane) : 0;
          const int lb = __shfl_sync(FULL, head, 0);
          const i32 bv = __shfl_down_sync(FULL, head, 1);  // entry `lane` (lanes < 31)
          if (lane < lb && lane < 31) {
            const i32 e = bv - D.rb;
            sm_red_xor32(D.bits + (e >> 5), 1u << (e & 31));
          }
          if (lb > 31) dense_flip(D, pool + at_f + 32, true, lb - 31, D.rb);
          __syncwarp();
          ++n_merges;
          published = false;
          // the added record cleared the old pivot: the new one is the first set
          // bit from its word on, almost always within the next 32 words
          const i64 wp = (i64)((pf - D.rb) >> 5);
          const i64 wl = wp + lane;
          const u32 v = wl < dwords ? sm_ld32(D.bits + wl) : 0u;
          const u32 m = __ballot_sync(FULL, v != 0);
          i32 np;
          if (m) {
            const int f = __ffs(m) - 1;
            const u32 vw = __shfl_sync(FULL, v, f);
            np = (i32)(((wp + f) << 5) + (__ffs(vw) - 1)) + D.rb;
          } else {
            np = dense_first(D, wp + 32, D.rb);
          }
          D.piv = np;
          if (np < 0) break;
          if (++step >= max_steps) break;
          if ((step & 63) == 63 && *vabort) {
            aborted = true;
            break;
          }
        }
        if (aborted) break;
        if (D.piv < 0) {  // the column vanished
          k = 0;
          leave_dense();
          break;
        }
        if (!have_ow) continue;  // the step limit: the loop top reports it
      }
      const i32 p = dense ? D.piv : (wg ? __ldcg(W) : W[0]);
      u64 ow = take ? pending : (have_ow ? ow_known : ld_acquire(owner + (p - row_base)));
      pending = 0;
      i32 o = owner_col(ow);
      if (!take && o < c) {
        // publish W as a record, then claim p
        if (!published) {
          if (dense) k = dense_count(D, D.rb);
          const unsigned long long at = pool_alloc(chunk_state, ctl, pool_cap, k + 1, chunk, status);
          if (at == ~0ull) break;
          if (lane == 0) pool[at] = k;
          if (dense)
            dense_to_list(D, D.rb, pool + at + 1);
          else
            for (int i = lane; i < k; i += 32) pool[at + 1 + i] = wg ? __ldcg(W + i) : W[i];
          wrec = at;
          published = true;
        }
        __syncwarp();
        u64 old = 0;
        if (lane == 0) old = atom_max_acq_rel(owner + (p - row_base), owner_word(c, wrec));
        old = __shfl_sync(FULL, old, 0);
        __syncwarp();
        const i32 oc = owner_col(old);
        if (oc < c) {
          if (oc < 0) {  // claimed a free pivot: this work item is done
            leave_dense();
            break;
          }
          // displaced a smaller column: take it over
          ++n_takeovers;
          c = oc;
          if (dense) {
            // the bitmap holds the claimer's content: flip the displaced record into it
            const u64 at_d = old & OW_OFF;
            const int len_d = __ldcg(pool + at_d);
            dense_flip(D, pool + at_d + 1, true, len_d, D.rb);
            ++n_merges;
            published = false;
            D.piv = dense_first(D, (i64)((p - D.rb) >> 5), D.rb);
            if (D.piv < 0) {  // the column vanished
              k = 0;
              leave_dense();
              break;
            }
            k = 1;  // nonzero; counted when published
            continue;
          }
          if (!wg) {
            pending = old;  // next step: W (the claimer's content) + the displaced record
            continue;
          }
          load_record(old & OW_OFF);
          continue;
        }
        o = oc;  // a larger column got there first
        ow = old;
      }
      if (!take && o == c) {  // cannot happen: a column never owns a pivot it is still reducing
        if (lane == 0) set_status(status, PH_ERR_ARG);
        break;
      }
      // add the larger owner o: its record head (length + 31 entries) in one load
      const u64 at_o = ow & OW_OFF;
      const i32 head = (at_o + lane < (u64)pool_cap) ? __ldcg(pool + at_o + lane) : 0;
      const int lb = __shfl_sync(FULL, head, 0);
      const i32 bv = __shfl_down_sync(FULL, head, 1);  // entry `lane` of B (lanes < 31)
      if (!dense && dense_ok && k + lb > RD_CAP) enter_dense(W, wg, k);  // W outgrows its buffer
      if (dense) {
        // entries 0..30 of the added column are already in registers
        if (lb <= 31)
          dense_flip_regs(D, bv, lb, D.rb);
        else
          dense_flip(D, pool + at_o + 1, true, lb, D.rb);
        ++n_merges;
        published = false;
        D.piv = dense_first(D, (i64)((p - D.rb) >> 5), D.rb);
        if (D.piv < 0) {  // the column vanished
          k = 0;
          leave_dense();
          break;
        }
        k = 1;  // nonzero; counted when published
        continue;
      }
      if (!wg && lb <= 31 && k + lb <= RD_CAP) {
        const int m = warp_xor_small<false>(W, k, lane < lb ? bv : INT_MAX, lb, (sW0 + (cur ^ 1) * RD_CAP));
        __syncwarp();
        ++n_merges;
        k = m;
        cur ^= 1;
        W = (sW0 + cur * RD_CAP);
        published = false;
        continue;
      }
      const i32* Bsrc = pool + at_o + 1;
      const i32* B;
      bool bg;
      if (lb <= RD_CAPB) {
        if (lane < 31 && lane < lb) sBw[lane] = bv;
        for (int i = 31 + lane; i < lb; i += 32) sBw[i] = __ldcg(Bsrc + i);
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
        out = (sW0 + (cur ^ 1) * RD_CAP);
        og = false;
      } else {
        at = pool_alloc(chunk_state, ctl, pool_cap, k + lb + 1, chunk, status);
        if (at == ~0ull) break;
        out = pool + at + 1;
        og = true;
      }
      const int m = symdiff(W, wg, k, B, bg, lb, out);
      __syncwarp();
      ++n_merges;
      k = m;
      if (og) {
        if (lane == 0) pool[at] = m;
        __syncwarp();
        W = out;
        wg = true;
        wrec = at;
        published = true;
      } else {
        cur ^= 1;
        W = (sW0 + cur * RD_CAP);
        wg = false;
        published = false;
      }
    }
    leave_dense();  // every exit leaves the slot clean for the next column
    }
  }
  if (lane == 0) {
    if (n_merges) atomicAdd(&ctl->merges, n_merges);
    if (n_takeovers) atomicAdd(&ctl->takeovers, n_takeovers);
  }
}

// residual columns default to empty (state 3) ...
__global__ void k_finish_cols(i64 K, i32* __restrict__ state, i32* __restrict__ piv, const RedCtl* ctl, i64* info) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x) {
    if (state[c] != 2) continue;
    state[c] = 3;
    piv[c] = -1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && info) {
    info[0] = ctl->nres;
    info[1] = (i64)ctl->merges;
    info[2] = (i64)ctl->pool_top;
    info[3] = (i64)ctl->takeovers;
  }
}

// ... and a residual column that owns a row at the end is paired with it
__global__ void k_finish_rows(const u64* __restrict__ owner, i64 R, i32 row_base, i32* __restrict__ state,
                              i32* __restrict__ piv) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < R; r += (i64)gridDim.x * blockDim.x) {
    const u64 w = owner[r];
    if (!w) continue;
    const i32 c = owner_col(w);
    if (state[c] == 1) continue;  // apparent
    state[c] = 2;
    piv[c] = (i32)r + row_base;
  }
}

__global__ void k_mark_pivots(const i32* __restrict__ state, const i32* __restrict__ piv, i64 K, i32 row_base,
                              uint8_t* __restrict__ flag) {
  ph::pdl_wait();
  ph::pdl_trigger();
  for (i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x; c < K; c += (i64)gridDim.x * blockDim.x)
    if (state[c] == 1 || state[c] == 2) flag[piv[c] - row_base] = 1;
}

inline int grid_for(i64 n, int nt = 256) {
  return (int)std::max<i64>(1, std::min<i64>((n + nt - 1) / nt, 148 * 16));
}

}  // namespace
}  // namespace ph

using namespace ph;

// Grid of k_reduce on the current device: persistent blocks, one per resident slot.
int reduce_blocks(i64 K) {
  ph::allow_dynamic_smem((const void*)k_reduce);
  const int sms = ph::device_sms();
  const int occ = ph::occupancy((const void*)k_reduce, RD_NT, RD_SMEM);
  return (int)std::max<i64>(1, std::min<i64>((K + RD_WARPS - 1) / RD_WARPS, (i64)sms * std::max(occ, 1)));
}

// A dense working column's bitmap starts at the word of its first pivot and
// must hold every row its entries can reach: `span` rows (all R rows for a
// single cloud; in a batch, the largest row range of one cloud, since a
// column only ever meets rows of its own cloud), plus a word of alignment,
// rounded up to whole 32-word blocks (slots and blocks 128-byte aligned).
i64 window_words(i64 span) { return ((span + 31) / 32 + 2 + 31) / 32 * 32; }

// words of the shared-memory bitmap each warp uses for every working column,
// 0 when the window does not fit one working buffer
int sm_dense_words(i64 span) {
  const i64 words = window_words(span);
  return words <= RD_CAP ? (int)words : 0;
}

// dense working-column slots in global memory (windows beyond the shared
// bitmap): one window per warp of the grid, when they fit in 1 GiB (else long
// columns stay sorted lists in the pool)
i64 dense_words(i64 K, i64 span) {
  if (sm_dense_words(span)) return 0;
  const i64 words = window_words(span);
  const i64 warps = (i64)reduce_blocks(K) * RD_WARPS;
  return words * warps * 4 <= (i64(1) << 30) ? words : 0;
}

inline i64 span_or_all(i64 R, i64 span) { return span > 0 && span < R ? span : R; }

extern "C" size_t ph_reduce_workspace_bytes(int64_t K, int64_t R, int64_t span) {
  span = span_or_all(R, span);
  const i64 dw = K > 0 ? dense_words(K, span) : 0;
  return Carve::need((size_t)R * 8) + Carve::need((size_t)K * 8) + Carve::need(sizeof(RedCtl)) +
         (dw ? Carve::need((size_t)dw * 4 * reduce_blocks(K) * RD_WARPS) : 0);
}

extern "C" int ph_reduce(const int32_t* cof_off, const int32_t* cof_data, int64_t K, int32_t col_base,
                         int64_t R, int32_t row_base, int64_t span, const uint8_t* skip, const int32_t* row_cmf,
                         int32_t* col_state, int32_t* col_piv, int32_t* pool, int64_t pool_cap,
                         int64_t* d_info, int* d_status, void* workspace, size_t workspace_bytes,
                         void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0 || R < 0 || pool_cap < 0) return PH_ERR_ARG;
  if (K >= (int64_t(1) << 31) || R >= (int64_t(1) << 31) || pool_cap >= (int64_t(1) << OW_SHIFT))
    return PH_ERR_OVERFLOW;
  if (K == 0) {
    if (d_info) ph::zero_async(d_info, 4 * sizeof(int64_t), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  Carve c(workspace, workspace_bytes);
  u64* owner = c.take<u64>(std::max<i64>(R, 1));
  u64* rec = c.take<u64>(K);
  RedCtl* ctl = c.take<RedCtl>(1);
  if (!owner || !rec || !ctl) return PH_ERR_ARG;
  ph::zero_async(owner, sizeof(u64) * std::max<i64>(R, 1), s, ctl, sizeof(RedCtl));
  ph::count_launch();
  ph::launch_pdl(k_classify, dim3(grid_for(K)), dim3(256), 0, s, cof_off, cof_data, K, col_base, row_base, skip, row_cmf, col_state,
                                         col_piv, owner, rec, pool, pool_cap, ctl, d_status);
  if (ph::allow_dynamic_smem((const void*)k_reduce) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  const int blocks = reduce_blocks(K);
  span = span_or_all(R, span);
  const i64 dw = dense_words(K, span);
  u32* dense = dw ? c.take<u32>(dw * (i64)blocks * RD_WARPS) : nullptr;
  if (dw && !dense) return PH_ERR_ARG;
  // pool chunk per warp: small enough that the chunks of all warps fit a quarter of the pool
  const int chunk = (int)std::max<i64>(64, std::min<i64>(2048, pool_cap / (4 * (i64)blocks * RD_WARPS)));
  ph::count_launch();
  ph::launch_pdl(k_reduce, dim3(blocks), dim3(RD_NT), RD_SMEM, s, row_base, K, col_state, rec, owner, pool, pool_cap, chunk, ctl, d_status,
                                          (int)std::min<long long>(ph::reduce_max_steps(), INT_MAX), dense, dw,
                                          sm_dense_words(span));
  ph::count_launch();
  ph::launch_pdl(k_finish_cols, dim3(grid_for(K)), dim3(256), 0, s, K, col_state, col_piv, ctl, d_info);
  if (R > 0) {
    ph::count_launch();
    ph::launch_pdl(k_finish_rows, dim3(grid_for(R)), dim3(256), 0, s, owner, R, row_base, col_state, col_piv);
  }
  PH_CHECK_LAUNCH();
  return PH_OK;
}

extern "C" int ph_mark_pivots(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                              uint8_t* row_flag, int64_t R, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (K < 0 || R < 0) return PH_ERR_ARG;
  if (R > 0) ph::zero_async(row_flag, (size_t)R, s);
  if (K > 0) {
    ph::count_launch();
    ph::launch_pdl(k_mark_pivots, dim3(grid_for(K)), dim3(256), 0, s, col_state, col_piv, K, row_base, row_flag);
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
