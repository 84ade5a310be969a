// Edge enumeration with a tensor-core screen (the precision form).
//
// The reference's kernel (kernels/edge_kernel.py:23-149) spends 2d FP32
// instructions per pair. Here pairs are first screened with a BF16 Gram
// product on the 5th-generation tensor cores, and only the pairs that pass
// are recomputed with the exact FP32 chain of ph_edges_enumerate
// (df = x_k - y_k; acc = fma(df, df, acc), k ascending), so the edge set and
// every dist^2 bit are those of the direct kernel.
//
// Screen. Each cloud is centred on its mean mu (FP64) and rounded to BF16:
// y^_i = bf16(x_i - mu). With n_i = |y^_i|^2 (FP64, exact products) and
// a'_i <= (1 - kappa) n_i a 16-bit lower bound held as two BF16 parts, the
// operands are augmented by four K columns
//     A row i = [ y^_i,   ah_i, al_i, 1,    1    ]
//     B row j = [ -2y^_j, 1,    1,    ah_j, al_j ]
// so one tcgen05.mma chain (M = N = 128, FP32 accumulation in TMEM) yields
//     S_ij = a'_i + a'_j - 2 <y^_i, y^_j>
// directly, and the epilogue is one compare per pair.
//
// Certificate (per pair i < j, u = 2^-24):
//   - exact chain C < thr  =>  true D = |x_i - x_j|^2 < thr (1 + (d + 3) u)
//     (one rounding per subtraction and per fma);
//   - centring is a translation by the same real mu, so differences are
//     exact; BF16 rounding (unit roundoff 2^-8, also after a rounding of
//     the FP64 difference) moves each point by at most
//     r_i = 1.01 * 2^-8 |y^_i| + sqrt(d) 2^-120 (the last term covers BF16
//     and FP32 values flushed to zero), so sqrt(D^) <= sqrt(D) + r_i + r_j
//     for D^ = |y^_i - y^_j|^2 = n_i + n_j - 2 G_ij;
//   - the MMA's products are exact; its FP32 accumulation is assumed to err
//     by at most (kappa / 2) sum |terms| <= kappa (n_i + n_j), kappa =
//     max(2^-11, K 2^-18) for K accumulated columns: at least 12 correct
//     bits against the sum of magnitudes, where measurements of BF16 MMA
//     accumulation show about 23. Then S <= D^.
// Hence C < thr implies S < (sqrt(thr (1 + (d+3)u)) + r_i + r_j)^2, which the
// screen tests against the per-tile maxima of r (rounded up, plus 2^-20
// relative and 2^-96 absolute). A tile whose widened threshold is not finite
// (non-finite or huge points, |y^|^2 >= 2^120, or a huge threshold) skips
// the screen and recomputes every pair exactly.
//
// Kernel anatomy (one CTA = 4 warps, persistent over 128 x 128 point tiles):
//   all threads : copy both BF16 operand tiles into shared memory in the
//                 128-byte-swizzled K-major layout the UMMA descriptors name
//   thread 0    : ceil((d + 4) / 16) tcgen05.mma (K = 16 each) into TMEM,
//                 tcgen05.commit to an mbarrier, bounded wait on it
//   warp w      : tcgen05.ld of TMEM lanes 32w..32w+31 (its 32 rows), one
//                 compare + ballot per column, candidates compacted into a
//                 per-warp shared queue, then the exact chain for the queue
//                 with all 32 lanes busy and warp-aggregated emission
// TMEM: 128 columns per CTA; the dynamic shared memory request keeps at most
// three CTAs per SM (384 of the 512 columns).
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int TC_T = 128;          // tile side (points)
constexpr int TC_NT = 128;         // threads per CTA (4 warps)
constexpr int TC_KATOM = 64;       // BF16 elements per 128-byte swizzle atom row
constexpr int TC_ATOM_BYTES = TC_T * 128;
constexpr int TC_MAXK = 256;       // augmented K supported (d <= 252)
constexpr int TC_AUG = 4;          // augmented columns
constexpr int TC_QCAP = 32 * TC_T; // candidate slots per warp (all its pairs)
constexpr unsigned FULL = 0xffffffffu;
constexpr int TC_WAIT_LIMIT = 1 << 26;

__host__ __device__ inline int tc_kq(int d) { return ((d + TC_AUG + 15) / 16) * 16; }

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ int find_off(const i64* off, int nsegs, i64 b) {
  int lo = 0, hi = nsegs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int find_seg_tc(const ph_cloud_seg* segs, int nsegs, i64 b) {
  int lo = 0, hi = nsegs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].tile_off <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// upper-triangular tile b of an nt x nt grid, row-major (same order as ph_edges_enumerate)
__device__ __forceinline__ void tile_coords_tc(i64 b, i64 nt, i64& I, i64& J) {
  const double a = 2.0 * (double)nt + 1.0;
  i64 r = (i64)floor((a - sqrt(a * a - 8.0 * (double)b)) * 0.5);
  if (r < 0) r = 0;
  auto start = [nt](i64 x) { return x * nt - x * (x - 1) / 2; };
  while (r > 0 && start(r) > b) --r;
  while (start(r + 1) <= b) ++r;
  I = r;
  J = r + (b - start(r));
}

// ---- prep: centre, round to BF16, augment --------------------------------------------
// sum of coordinates per cloud, FP64, from per-block partial sums (block = 128 points)
__global__ void k_tc_mean(const float* __restrict__ pts, const ph_cloud_seg* __restrict__ segs, int nsegs,
                          const i64* __restrict__ blk_off, double* __restrict__ sum) {
  __shared__ double part[TC_MAXK];
  const i64 b = blockIdx.x;
  const int c = find_off(blk_off, nsegs, b);
  const ph_cloud_seg sg = segs[c];
  const i64 p0 = (b - blk_off[c]) * TC_T;
  for (int k = threadIdx.x; k < sg.d; k += blockDim.x) part[k] = 0.0;
  __syncthreads();
  for (int idx = threadIdx.x; idx < TC_T * sg.d; idx += blockDim.x) {
    const i64 p = p0 + idx / sg.d;
    if (p < sg.n) atomicAdd(&part[idx % sg.d], (double)pts[sg.pt_off + p0 * sg.d + idx]);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < sg.d; k += blockDim.x) atomicAdd(&sum[(i64)c * TC_MAXK + k], part[k]);
}

__global__ void k_tc_points(const float* __restrict__ pts, const ph_cloud_seg* __restrict__ segs, int nsegs,
                            const i64* __restrict__ blk_off, const double* __restrict__ sum, int kq, double kappa,
                            __nv_bfloat16* __restrict__ YA, __nv_bfloat16* __restrict__ YB,
                            float* __restrict__ rad) {
  const i64 b = blockIdx.x;
  const int c = find_off(blk_off, nsegs, b);
  const ph_cloud_seg sg = segs[c];
  const i64 p = (b - blk_off[c]) * TC_T + threadIdx.x;
  if (p >= sg.n) return;
  const int d = sg.d;
  const double inv_n = 1.0 / (double)sg.n;
  const float* x = pts + sg.pt_off + p * d;
  __nv_bfloat16* ya = YA + (sg.vbase + p) * kq;
  __nv_bfloat16* yb = YB + (sg.vbase + p) * kq;
  double nrm = 0.0;
  for (int k = 0; k < d; ++k) {
    const double mu = sum[(i64)c * TC_MAXK + k] * inv_n;
    const __nv_bfloat16 v = __double2bfloat16((double)x[k] - mu);
    const float vf = __bfloat162float(v);
    nrm += (double)vf * (double)vf;
    ya[k] = v;
    yb[k] = __float2bfloat16_rn(-2.0f * vf);  // exact: a power-of-two scaling
  }
  const bool bad = !(nrm < 0x1p120);  // NaN, infinite or huge: the tile is recomputed exactly
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f), one = __float2bfloat16_rn(1.0f);
  if (bad) {
    for (int k = 0; k < d; ++k) ya[k] = yb[k] = zero;
    nrm = 0.0;
  }
  const float af = __double2float_rd((1.0 - kappa) * nrm);
  const __nv_bfloat16 ah = __float2bfloat16_rd(af);
  const __nv_bfloat16 al = __float2bfloat16_rd(af - __bfloat162float(ah));  // af - ah is exact
  ya[d] = ah;
  ya[d + 1] = al;
  ya[d + 2] = one;
  ya[d + 3] = one;
  yb[d] = one;
  yb[d + 1] = one;
  yb[d + 2] = ah;
  yb[d + 3] = al;
  for (int k = d + TC_AUG; k < kq; ++k) ya[k] = yb[k] = zero;
  rad[sg.vbase + p] =
      bad ? INFINITY : __double2float_ru(1.01 * 0x1p-8 * sqrt(nrm) + sqrt((double)d) * 0x1p-120);
}

// ---- tcgen05 helpers -------------------------------------------------------------------
__device__ __forceinline__ u64 umma_desc_sw128(u32 saddr) {
  // K-major, 128-byte swizzle: start >> 4, LBO = 1 (unused for this layout),
  // SBO = 1024 B (8-row group stride) >> 4, version 1 (bits 46-47),
  // layout type 2 = SWIZZLE_128B (bits 61-63), base offset 0 (1 KB aligned atoms)
  u64 d = 0;
  d |= (u64)((saddr >> 4) & 0x3fff);
  d |= (u64)1 << 16;
  d |= (u64)64 << 32;
  d |= (u64)1 << 46;
  d |= (u64)2 << 61;
  return d;
}

__device__ __forceinline__ u32 umma_idesc_bf16_f32(int M, int N) {
  u32 d = 0;
  d |= 1u << 4;              // C format F32
  d |= 1u << 7;              // A format BF16
  d |= 1u << 10;             // B format BF16
  d |= (u32)(N >> 3) << 17;  // N >> 3
  d |= (u32)(M >> 4) << 24;  // M >> 4
  return d;                  // K-major A and B, no negation, dense
}

__device__ __forceinline__ void umma_bf16(u32 tmem_d, u64 da, u64 db, u32 idesc, u32 accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(u32 mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(u32 mbar, u32 parity) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void tmem_ld32(u32 taddr, float (&v)[32]) {
  u32 r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
        "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
        "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// the exact FP32 chain of ph_edges_enumerate
__device__ __forceinline__ float exact_dsq(const float* __restrict__ x, const float* __restrict__ y, int d) {
  float acc = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float df = __fsub_rn(__ldg(x + k), __ldg(y + k));
    acc = __fmaf_rn(df, df, acc);
  }
  return acc;
}

// warp-aggregated append of the lanes with emit set
__device__ __forceinline__ void emit_warp(bool emit, i64 gi, i64 gj, float acc, int lane, i32* __restrict__ oi,
                                          i32* __restrict__ oj, float* __restrict__ od, i64 cap,
                                          unsigned long long* __restrict__ count) {
  const u32 m = __ballot_sync(FULL, emit);
  if (m == 0) return;
  const int leader = __ffs(m) - 1;
  unsigned long long pos0 = 0;
  if (lane == leader) pos0 = atomicAdd(count, (unsigned long long)__popc(m));
  pos0 = __shfl_sync(FULL, pos0, leader);
  if (emit) {
    const unsigned long long pos = pos0 + __popc(m & lanemask_lt());
    if (pos < (unsigned long long)cap) {
      oi[pos] = (i32)gi;
      oj[pos] = (i32)gj;
      od[pos] = acc;
    }
  }
}

// ---- main kernel ------------------------------------------------------------------------
// dynamic shared memory (1 KB aligned): [A tile: natoms x 16 KB][B tile: natoms x 16 KB]
//                                       [4 warp queues x TC_QCAP u16]
__global__ void __launch_bounds__(TC_NT, 1)
    k_tc_edges(const float* __restrict__ pts_all, const ph_cloud_seg* __restrict__ segs, int nsegs, i64 ntiles,
               const __nv_bfloat16* __restrict__ YA, const __nv_bfloat16* __restrict__ YB,
               const float* __restrict__ rad, int kq, double thr_scale, i32* __restrict__ oi,
               i32* __restrict__ oj, float* __restrict__ od, i64 cap, unsigned long long* __restrict__ count,
               int* status, unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ u32 tmem_base_sh;
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ float red[2][4];
  __shared__ int wait_failed;
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int natoms = (kq + TC_KATOM - 1) / TC_KATOM;
  unsigned char* tA = smem;
  unsigned char* tB = smem + natoms * TC_ATOM_BYTES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned short* queue = reinterpret_cast<unsigned short*>(tB + natoms * TC_ATOM_BYTES) + warp * TC_QCAP;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const u32 tmem = tmem_base_sh;
  const u32 mbar_addr = smem_u32(&mbar);
  const u32 idesc = umma_idesc_bf16_f32(TC_T, TC_T);
  const int cpr = kq / 8;  // 16-byte chunks per operand row
  const int row = warp * 32 + lane;
  u32 phase = 0;
  bool failed = false;

  for (i64 b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const ph_cloud_seg sg = segs[find_seg_tc(segs, nsegs, b)];
    const i64 n = sg.n;
    const int d = sg.d;
    const i64 nt = (n + TC_T - 1) / TC_T;
    i64 I, J;
    tile_coords_tc(b - sg.tile_off, nt, I, J);
    const i64 i0 = I * TC_T, j0 = J * TC_T;
    // operand tiles: row r, 16-byte chunk q of atom a at a*16KB + r*128 + ((q ^ (r&7)) << 4)
    for (int idx = threadIdx.x; idx < TC_T * cpr; idx += TC_NT) {
      const int r = idx / cpr;
      const int ch = idx - r * cpr;
      const int a = ch >> 3, q = ch & 7;
      const int so = a * TC_ATOM_BYTES + r * 128 + ((q ^ (r & 7)) << 4);
      uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
      if (i0 + r < n) va = __ldg(reinterpret_cast<const uint4*>(YA + (sg.vbase + i0 + r) * kq) + ch);
      if (j0 + r < n) vb = __ldg(reinterpret_cast<const uint4*>(YB + (sg.vbase + j0 + r) * kq) + ch);
      *reinterpret_cast<uint4*>(tA + so) = va;
      *reinterpret_cast<uint4*>(tB + so) = vb;
    }
    {
      float ma = (i0 + row < n) ? rad[sg.vbase + i0 + row] : 0.0f;
      float mb = (j0 + row < n) ? rad[sg.vbase + j0 + row] : 0.0f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ma = fmaxf(ma, __shfl_xor_sync(FULL, ma, o));
        mb = fmaxf(mb, __shfl_xor_sync(FULL, mb, o));
      }
      if (lane == 0) {
        red[0][warp] = ma;
        red[1][warp] = mb;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // widened squared threshold of this tile (identical in every thread)
    const float rA = fmaxf(fmaxf(red[0][0], red[0][1]), fmaxf(red[0][2], red[0][3]));
    const float rB = fmaxf(fmaxf(red[1][0], red[1][1]), fmaxf(red[1][2], red[1][3]));
    const double radius = sqrt((double)sg.thr_sq * thr_scale) + (double)rA + (double)rB;
    const double base_d = radius * radius * (1.0 + 0x1p-20) + 0x1p-96;
    const bool force = !(base_d < 3.0e38);
    const float base = force ? 0.0f : __double2float_ru(base_d);
    const float* P = pts_all + sg.pt_off;
    const i64 gi = i0 + row;

    if (!force) {
      if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int ks = (d + TC_AUG + 15) / 16;
        for (int s = 0; s < ks; ++s) {
          const int a = s >> 2, k = s & 3;
          const u64 da = umma_desc_sw128(smem_u32(tA + a * TC_ATOM_BYTES)) + (u64)(k * 2);
          const u64 db = umma_desc_sw128(smem_u32(tB + a * TC_ATOM_BYTES)) + (u64)(k * 2);
          umma_bf16(tmem, da, db, idesc, s > 0 ? 1u : 0u);
        }
        umma_commit(mbar_addr);
        int spins = 0;
        bool ok = true;
        while (!mbar_try_wait(mbar_addr, phase)) {
          if (++spins > TC_WAIT_LIMIT) {
            ok = false;
            break;
          }
        }
        wait_failed = ok ? 0 : 1;
        if (!ok) set_status(status, PH_ERR_ITER_LIMIT);
      }
      __syncthreads();
      if (wait_failed) {
        failed = true;
        break;
      }
      phase ^= 1;
      asm volatile("tcgen05.fence::after_thread_sync;");
      // screen: one compare per pair, candidates into this warp's queue
      int cnt = 0;
      const u32 lt = lanemask_lt();
      for (int c0 = 0; c0 < TC_T; c0 += 32) {
        float g[32];
        tmem_ld32(tmem + ((u32)(warp * 32) << 16) + (u32)c0, g);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const bool pass = g[k] < base;
          const u32 m = __ballot_sync(FULL, pass);
          if (m) {
            if (pass) queue[cnt + __popc(m & lt)] = (unsigned short)((row << 7) | (c0 + k));
            cnt += __popc(m);
          }
        }
      }
      __syncwarp();
      if (stats && lane == 0 && cnt) atomicAdd(&stats[0], (unsigned long long)cnt);
      // exact chain for the candidates, 32 at a time
      for (int e0 = 0; e0 < cnt; e0 += 32) {
        const int e = e0 + lane;
        bool emit = false;
        float acc = 0.0f;
        i64 qi = 0, qj = 0;
        if (e < cnt) {
          const u32 en = queue[e];
          qi = i0 + (en >> 7);
          qj = j0 + (en & 127);
          if (qi < qj && qj < n) {
            acc = exact_dsq(P + qi * d, P + qj * d, d);
            emit = acc < sg.thr_sq;
          }
        }
        emit_warp(emit, sg.vbase + qi, sg.vbase + qj, acc, lane, oi, oj, od, cap, count);
      }
      __syncwarp();
    } else {
      // no screen for this tile: every pair exactly
      if (stats && threadIdx.x == 0) atomicAdd(&stats[1], (unsigned long long)(TC_T * TC_T));
      for (int col = 0; col < TC_T; ++col) {
        const i64 gj = j0 + col;
        bool emit = false;
        float acc = 0.0f;
        if (gi < gj && gj < n) {
          acc = exact_dsq(P + gi * d, P + gj * d, d);
          emit = acc < sg.thr_sq;
        }
        emit_warp(emit, sg.vbase + gi, sg.vbase + gj, acc, lane, oi, oj, od, cap, count);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  // a failed wait: give the MMAs time to drain (bounded) before freeing TMEM
  if (failed && threadIdx.x == 0) {
    int spins = 0;
    while (!mbar_try_wait(mbar_addr, phase) && ++spins < TC_WAIT_LIMIT) {
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

}  // namespace
}  // namespace ph

using namespace ph;

namespace {

struct TcPlan {
  int kq, natoms;
  size_t smem;
};

TcPlan plan_for(int max_d) {
  TcPlan p;
  p.kq = tc_kq(max_d);
  p.natoms = (p.kq + TC_KATOM - 1) / TC_KATOM;
  // operand tiles + candidate queues + 1 KB alignment slack (>= 65 KB: at most
  // three CTAs, 384 TMEM columns, per SM)
  p.smem = (size_t)p.natoms * 2 * TC_ATOM_BYTES + (size_t)4 * TC_QCAP * 2 + 1024;
  return p;
}

}  // namespace

extern "C" size_t ph_edges_screened_workspace_bytes(int64_t N, int32_t nsegs, int32_t max_d) {
  if (N < 0 || nsegs < 1 || max_d < 1 || max_d > TC_MAXK - TC_AUG) return 0;
  const TcPlan p = plan_for(max_d);
  const size_t rows = (size_t)std::max<int64_t>(N, 1);
  return 2 * Carve::need(rows * p.kq * sizeof(__nv_bfloat16)) + Carve::need(rows * sizeof(float)) +
         Carve::need((size_t)nsegs * TC_MAXK * sizeof(double));
}

extern "C" int ph_batch_edges_enumerate_screened(const float* pts, const ph_cloud_seg* segs, int32_t nsegs,
                                                 int64_t ntiles, int32_t max_d, int64_t N, const int64_t* blk_off,
                                                 int64_t nblocks, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                                 int64_t capacity, unsigned long long* d_count, int* d_status,
                                                 unsigned long long* d_stats, void* workspace,
                                                 size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nsegs < 1 || ntiles < 0 || max_d < 1 || max_d > TC_MAXK - TC_AUG || N < 0 || capacity < 0 || !d_count ||
      !segs || !blk_off || nblocks < 0) {
    record_message("ph_batch_edges_enumerate_screened: invalid argument (d must be in [1, 252])");
    return PH_ERR_ARG;
  }
  if (ntiles >= (int64_t(1) << 31) || nblocks >= (int64_t(1) << 31) || N >= (int64_t(1) << 31))
    return PH_ERR_OVERFLOW;
  const TcPlan p = plan_for(max_d);
  const i64 rows = std::max<i64>(N, 1);
  Carve c(workspace, workspace_bytes);
  __nv_bfloat16* YA = c.take<__nv_bfloat16>(rows * p.kq);
  __nv_bfloat16* YB = c.take<__nv_bfloat16>(rows * p.kq);
  float* rad = c.take<float>(rows);
  double* sum = c.take<double>((i64)nsegs * TC_MAXK);
  if (!YA || !YB || !rad || !sum) {
    record_message("ph_batch_edges_enumerate_screened: workspace too small");
    return PH_ERR_ARG;
  }
  cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (ntiles == 0 || N == 0 || nblocks == 0) {
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  if (cudaFuncSetAttribute(k_tc_edges, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  int dev = 0, sms = 148, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tc_edges, TC_NT, p.smem);
  if (occ < 1 || occ * 128 > 512) {
    record_message("ph_batch_edges_enumerate_screened: unexpected occupancy for the TMEM budget");
    return PH_ERR_CUDA;
  }
  cudaMemsetAsync(sum, 0, sizeof(double) * nsegs * TC_MAXK, s);
  const double kappa = std::max(0x1p-11, (double)p.kq * 0x1p-18);
  ph::count_launch();
  k_tc_mean<<<(unsigned)nblocks, 256, 0, s>>>(pts, segs, nsegs, blk_off, sum);
  ph::count_launch();
  k_tc_points<<<(unsigned)nblocks, TC_T, 0, s>>>(pts, segs, nsegs, blk_off, sum, p.kq, kappa, YA, YB, rad);
  const double thr_scale = 1.0 + (double)(max_d + 3) * 0x1p-24;
  const int grid = (int)std::min<i64>(ntiles, (i64)sms * occ);
  ph::count_launch();
  k_tc_edges<<<grid, TC_NT, p.smem, s>>>(pts, segs, nsegs, ntiles, YA, YB, rad, p.kq, thr_scale, out_i, out_j,
                                         out_dsq, capacity, d_count, d_status, d_stats);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
