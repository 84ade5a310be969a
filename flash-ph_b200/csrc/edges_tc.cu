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
// Kernel anatomy (one persistent CTA per SM, 10 warps, a contiguous range of
// work items; an item is row block I (128 points) against column blocks
// J .. J + nb - 1, nb = 2 (MMA N = 256) unless the operand rings would not
// fit shared memory, rows in order, clipped at the cloud's last block):
//   warp 8 (producer) : TMA loads (cp.async.bulk.tensor, 2-D, swizzled, no
//                       multicast) of the A tile (row block I, reused while I
//                       is unchanged) and the B tile (column block J) into
//                       shared-memory rings, completion on mbarriers
//   warp 9 (MMA)      : one thread issues ceil((d + 4) / 16) tcgen05.mma
//                       (M = N = 128, K = 16) into one of two TMEM
//                       accumulator stages, tcgen05.commit frees the operand
//                       stages and publishes the accumulator
//   warps 0-7         : two warpgroups taking alternate tiles (one TMEM
//                       stage each); a warp reads its 32 TMEM lanes x 128
//                       columns (two tcgen05.ld in flight), a min pre-check
//                       then one compare + ballot per column, candidates
//                       compacted into a per-warp queue that spans tiles and
//                       is recomputed with the exact chain 32 pairs at a
//                       time, with warp-aggregated emission
// Each cloud's operand rows are padded to a multiple of 128 with rows whose
// augmented columns carry 2^100, so padding never passes the screen. Every
// wait is bounded (a few seconds of global time); a timeout sets
// PH_ERR_ITER_LIMIT, stops every role, and the in-flight copies and MMAs are
// drained (again bounded) before TMEM is freed.
#include <algorithm>
#include <cmath>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "prim.cuh"

namespace ph {
namespace {

constexpr int TC_T = 128;                 // tile side (points)
constexpr int TC_MAXK = 256;              // augmented K supported (d <= 252)
constexpr int TC_AUG = 4;                 // augmented columns
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_PRODUCER_WARP = 8;
constexpr int TC_MMA_WARP = 9;
constexpr int TC_THREADS = 320;
constexpr int TC_QCAP = 512;              // candidate pairs queued per epilogue warp (across tiles)
constexpr int TC_MAX_STAGES = 6;
constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned long long TC_WAIT_NS = 4000000000ull;
constexpr float TC_PAD_NORM = 0x1p100f;   // augmented value of padding rows

// operand geometry fixed per launch
struct TcShape {
  int kq;            // K columns of an operand row: 16, 32 or a multiple of 64
  int box_k;         // K columns per TMA box and swizzle row: min(kq, 64)
  int natoms;        // K atoms (TMA boxes along K) per operand
  int row_bytes;     // box_k x 2
  int nb;            // 128-point column blocks per work item (1 or 2: MMA N = 128 nb)
  int a_atom_bytes;  // 128 rows x row_bytes
  int b_atom_bytes;  // 128 nb rows x row_bytes
  int a_bytes;       // natoms x a_atom_bytes
  int b_bytes;       // natoms x b_atom_bytes
  int ns, na;        // B and A ring stages
  u32 layout;        // UMMA layout type: 6 = 32-byte, 4 = 64-byte, 2 = 128-byte swizzle
  u32 sbo;           // 8-row group stride (8 x row_bytes) >> 4
};

__host__ __device__ inline int tc_kq(int d) {
  const int k = d + TC_AUG;
  return k <= 16 ? 16 : k <= 32 ? 32 : ((k + 63) / 64) * 64;
}

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

// Work items of a cloud with nt 128-point blocks: row block I against column
// blocks J .. J + nb - 1 (clipped at nt), J = I, I + nb, ...; rows in order.
// items(I) = ceil((nt - I) / nb); rows_before(I) = sum of items(r), r < I.
__host__ __device__ inline i64 tc_rows_before(i64 I, i64 nt, int nb) {
  if (nb == 1) return I * nt - I * (I - 1) / 2;
  auto F = [](i64 M) { return (M & 1) ? ((M + 1) / 2) * ((M + 1) / 2) : (M / 2) * (M / 2 + 1); };
  return F(nt) - F(nt - I);
}

__host__ __device__ inline i64 tc_cloud_items(i64 n, int nb) {
  if (n < 2) return 0;
  const i64 nt = (n + TC_T - 1) / TC_T;
  return tc_rows_before(nt, nt, nb);
}

// walks the global item sequence: clouds in table order, rows I, column blocks J
struct ItemIt {
  const ph_cloud_seg* segs;
  const i64* blk_off;
  const i64* item_off;
  int nsegs, nb, c;
  i64 I, J, nt, blk;
  ph_cloud_seg sg;
  __device__ int nh() const { return (nt - J) < nb ? (int)(nt - J) : nb; }  // column blocks in this item
  __device__ bool row_end() const { return J + nb >= nt; }
  __device__ void load() {
    sg = segs[c];
    nt = (sg.n + TC_T - 1) / TC_T;
    blk = blk_off[c];
  }
  __device__ void start(i64 q) {
    // clouds without items share their successor's offset; take the last such entry
    int lo = 0, hi = nsegs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (item_off[mid] <= q) lo = mid;
      else hi = mid - 1;
    }
    c = lo;
    load();
    const i64 local = q - item_off[c];
    i64 a = 0, b = nt - 1;  // largest I with rows_before(I) <= local
    while (a < b) {
      const i64 mid = (a + b + 1) >> 1;
      if (tc_rows_before(mid, nt, nb) <= local) a = mid;
      else b = mid - 1;
    }
    I = a;
    J = I + (i64)nb * (local - tc_rows_before(I, nt, nb));
  }
  // only called while another item exists
  __device__ void next() {
    J += nb;
    if (J < nt) return;
    if (++I < nt) {
      J = I;
      return;
    }
    do {
      ++c;
    } while (c < nsegs - 1 && segs[c].n < 2);
    load();
    I = J = 0;
  }
};

// item_off[c] = items of clouds before c, item_off[nsegs] = total (one block)
__global__ void k_tc_items(const ph_cloud_seg* __restrict__ segs, int nsegs, int nb, i64* __restrict__ item_off) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ i64 part[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int chunk = (nsegs + nt - 1) / nt;
  const int c0 = tid * chunk, c1 = min(nsegs, c0 + chunk);
  i64 sum = 0;
  for (int c = c0; c < c1; ++c) sum += tc_cloud_items(segs[c].n, nb);
  part[tid] = sum;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {  // inclusive scan
    const i64 v = tid >= o ? part[tid - o] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  i64 run = part[tid] - sum;
  for (int c = c0; c < c1; ++c) {
    item_off[c] = run;
    run += tc_cloud_items(segs[c].n, nb);
  }
  if (tid == nt - 1) item_off[nsegs] = part[tid];
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
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

// waits for the phase of the given parity; false after a timeout (which also
// raises the abort flag) or when another role has aborted
__device__ bool mbar_wait(u32 mbar, u32 parity, volatile int* abort_flag) {
  if (mbar_try_wait(mbar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (true) {
    if (mbar_try_wait(mbar, parity)) return true;
    if (abort_flag && *abort_flag) return false;
    if (gtimer() - t0 > TC_WAIT_NS) {
      if (abort_flag) *abort_flag = 1;
      return false;
    }
  }
}

__device__ __forceinline__ void mbar_init(u32 mbar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(u32 mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(u32 mbar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(u32 dst, const CUtensorMap* map, int x, int y, u32 mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<u64>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

// ---- prep: centre, round to BF16, augment --------------------------------------------
// sum of coordinates per cloud, FP64, from per-block partial sums (block = 128 points)
__global__ void k_tc_mean(const float* __restrict__ pts, const ph_cloud_seg* __restrict__ segs, int nsegs,
                          const i64* __restrict__ blk_off, double* __restrict__ sum) {
  ph::pdl_wait();
  ph::pdl_trigger();
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

__device__ __forceinline__ u32 bf16_bits(__nv_bfloat16 v) { return (u32)__bfloat16_as_ushort(v); }

// One thread per padded operand row (block b = 128 rows of one cloud). Row
// layout: A = [y, ah, al, 1, 1, 0...], B = [-2y, 1, 1, ah, al, 0...];
// padding rows A = [0, 2^100, 0, 1, 1, 0...], B = [0, 1, 1, 2^100, 0, 0...].
// blkrad[b] = the largest rounding radius of the block's points.
__global__ void k_tc_points(const float* __restrict__ pts, const ph_cloud_seg* __restrict__ segs, int nsegs,
                            const i64* __restrict__ blk_off, const double* __restrict__ sum, int kq, double kappa,
                            __nv_bfloat16* __restrict__ YA, __nv_bfloat16* __restrict__ YB,
                            float* __restrict__ blkrad) {
  ph::pdl_wait();
  ph::pdl_trigger();
  __shared__ float wmax[TC_T / 32];
  const i64 b = blockIdx.x;
  const int c = find_off(blk_off, nsegs, b);
  const ph_cloud_seg sg = segs[c];
  const i64 p = (b - blk_off[c]) * TC_T + threadIdx.x;
  const int d = sg.d;
  const double* mu_sum = sum + (i64)c * TC_MAXK;
  const double inv_n = 1.0 / (double)sg.n;
  const float* x = pts + sg.pt_off + p * d;
  const bool real = p < sg.n;
  double nrm = 0.0;
  if (real) {
    for (int k = 0; k < d; ++k) {
      const float vf = __bfloat162float(__double2bfloat16((double)x[k] - mu_sum[k] * inv_n));
      nrm += (double)vf * (double)vf;
    }
  }
  const bool bad = real && !(nrm < 0x1p120);  // NaN, infinite or huge: tiles recomputed exactly
  if (bad) nrm = 0.0;
  const float af = real ? __double2float_rd((1.0 - kappa) * nrm) : TC_PAD_NORM;
  const __nv_bfloat16 ah = __float2bfloat16_rd(af);
  const __nv_bfloat16 al = real ? __float2bfloat16_rd(af - __bfloat162float(ah)) : __float2bfloat16_rn(0.0f);
  const __nv_bfloat16 one = __float2bfloat16_rn(1.0f), zero = __float2bfloat16_rn(0.0f);
  uint4* ya = reinterpret_cast<uint4*>(YA + (b * TC_T + threadIdx.x) * kq);
  uint4* yb = reinterpret_cast<uint4*>(YB + (b * TC_T + threadIdx.x) * kq);
  for (int k0 = 0; k0 < kq; k0 += 8) {
    u32 wa[4], wb[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      u32 pa = 0, pb = 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = k0 + e + h;
        __nv_bfloat16 va = zero, vb = zero;
        if (k < d) {
          if (real && !bad) {
            va = __double2bfloat16((double)x[k] - mu_sum[k] * inv_n);
            vb = __float2bfloat16_rn(-2.0f * __bfloat162float(va));  // exact: a power-of-two scaling
          }
        } else if (k == d) {
          va = ah;
          vb = one;
        } else if (k == d + 1) {
          va = al;
          vb = one;
        } else if (k == d + 2) {
          va = one;
          vb = ah;
        } else if (k == d + 3) {
          va = one;
          vb = al;
        }
        pa |= bf16_bits(va) << (16 * h);
        pb |= bf16_bits(vb) << (16 * h);
      }
      wa[e >> 1] = pa;
      wb[e >> 1] = pb;
    }
    ya[k0 >> 3] = make_uint4(wa[0], wa[1], wa[2], wa[3]);
    yb[k0 >> 3] = make_uint4(wb[0], wb[1], wb[2], wb[3]);
  }
  float r = 0.0f;
  if (real) r = bad ? INFINITY : __double2float_ru(1.01 * 0x1p-8 * sqrt(nrm) + sqrt((double)d) * 0x1p-120);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(FULL, r, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) blkrad[b] = fmaxf(fmaxf(wmax[0], wmax[1]), fmaxf(wmax[2], wmax[3]));
}

// ---- tcgen05 helpers -------------------------------------------------------------------
// K-major shared-memory matrix descriptor: start >> 4, LBO = 1 (unused for
// swizzled K-major operands), SBO = 8-row group stride >> 4, version 1
// (bits 46-47), base offset 0 (1 KB aligned tiles), layout type (bits 61-63)
__device__ __forceinline__ u64 umma_desc(u32 saddr, u32 layout, u32 sbo) {
  u64 d = 0;
  d |= (u64)((saddr >> 4) & 0x3fff);
  d |= (u64)1 << 16;
  d |= (u64)sbo << 32;
  d |= (u64)1 << 46;
  d |= (u64)layout << 61;
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

__device__ __forceinline__ void tmem_ld32_issue(u32 taddr, u32 (&r)[32]) {
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
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// the exact FP32 chain of ph_edges_enumerate
__device__ __forceinline__ float exact_dsq(const float* __restrict__ x, const float* __restrict__ y, int d) {
  float acc = 0.0f;
#pragma unroll 8
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

// Exact chain for the first cnt queued cloud-local pairs of cloud qs, 32 at a
// time with warp-aggregated emission. Kept out of line: the screening loop
// around its call sites must stay small.
__device__ __noinline__ void flush_queue(const uint2* __restrict__ queue, int cnt, const ph_cloud_seg qs,
                                         const float* __restrict__ pts_all, i32* __restrict__ oi,
                                         i32* __restrict__ oj, float* __restrict__ od, i64 cap,
                                         unsigned long long* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
  const float* P = pts_all + qs.pt_off;
  for (int e0 = 0; e0 < cnt; e0 += 32) {
    const int e = e0 + lane;
    bool emit = false;
    float acc = 0.0f;
    i64 qi = 0, qj = 0;
    if (e < cnt) {
      const uint2 en = queue[e];
      qi = en.x;
      qj = en.y;
      if (qi < qj && qj < qs.n) {
        acc = exact_dsq(P + qi * qs.d, P + qj * qs.d, qs.d);
        emit = acc < qs.thr_sq;
      }
    }
    emit_warp(emit, qs.vbase + qi, qs.vbase + qj, acc, lane, oi, oj, od, cap, count);
  }
  __syncwarp();
}

// ---- main kernel ------------------------------------------------------------------------
// barrier slots: B full [0, 6), B empty [6, 12), A full [12, 14), A empty [14, 16),
// TMEM full [16, 18), TMEM empty [18, 20)
constexpr int BAR_BF = 0, BAR_BE = 6, BAR_AF = 12, BAR_AE = 14, BAR_TF = 16, BAR_TE = 18, BAR_N = 20;

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_tc_edges(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const float* __restrict__ pts_all, const ph_cloud_seg* __restrict__ segs, int nsegs,
               const i64* __restrict__ blk_off, const i64* __restrict__ item_off, const float* __restrict__ blkrad,
               TcShape sh, double thr_scale, i32* __restrict__ oi, i32* __restrict__ oj, float* __restrict__ od,
               i64 cap, unsigned long long* __restrict__ count, int* status, unsigned long long* __restrict__ stats) {
  ph::pdl_wait();
  ph::pdl_trigger();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long bars[BAR_N];
  __shared__ u32 tmem_sh;
  __shared__ int abort_sh;
  __shared__ unsigned long long st_sh[2];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = smem;
  unsigned char* sB = smem + sh.na * sh.a_bytes;
  uint2* qbase = reinterpret_cast<uint2*>(sB + sh.ns * sh.b_bytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const u32 bar0 = smem_u32(bars);
  auto bar = [bar0](int slot) { return bar0 + 8u * (u32)slot; };
  volatile int* abort_flag = &abort_sh;
  const u32 stage_cols = (u32)(TC_T * sh.nb);  // TMEM columns per accumulator stage

  // contiguous item range of this CTA
  const i64 nitems = item_off[nsegs];
  const i64 per = (nitems + gridDim.x - 1) / gridDim.x;
  const i64 b0 = (i64)blockIdx.x * per;
  const i64 T = b0 < nitems ? (per < nitems - b0 ? per : nitems - b0) : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_MAX_STAGES; ++s) {
      mbar_init(bar(BAR_BF + s), 1);
      mbar_init(bar(BAR_BE + s), 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(bar(BAR_AF + s), 1);
      mbar_init(bar(BAR_AE + s), 1);
      mbar_init(bar(BAR_TF + s), 1);
      mbar_init(bar(BAR_TE + s), TC_EPI_WARPS / 2);
    }
    abort_sh = 0;
    st_sh[0] = st_sh[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == TC_MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(2 * stage_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const u32 tmem = tmem_sh;

  if (T > 0 && warp == TC_PRODUCER_WARP) {
    if (lane == 0) {
      ItemIt it{segs, blk_off, item_off, nsegs, sh.nb};
      it.start(b0);
      // ring positions kept incrementally (no divisions on this thread); a_ph /
      // b_ph = (use + 1) & 1 for the current use of the stage, which is the
      // parity of the empty-barrier phase that frees it
      int u = -1, as = -1, bs = -1;
      u32 a_ph = 1, b_ph = 1;
      bool new_a = true;
      i64 t = 0;
      bool ok = true;
      for (; t < T; ++t) {
        if (t) {
          new_a = it.row_end();  // the row block (or the cloud) changes
          it.next();
        }
        if (new_a) {
          ++u;
          if (++as == sh.na) {
            as = 0;
            a_ph ^= 1;
          }
          if (u >= sh.na && !(ok = mbar_wait(bar(BAR_AE + as), a_ph, abort_flag))) break;
          mbar_expect_tx(bar(BAR_AF + as), (u32)sh.a_bytes);
          const int y = (int)(TC_T * (it.blk + it.I));
          for (int a = 0; a < sh.natoms; ++a)
            tma_load_2d(smem_u32(sA + as * sh.a_bytes + a * sh.a_atom_bytes), &tmA, a * 64, y, bar(BAR_AF + as));
        }
        if (++bs == sh.ns) {
          bs = 0;
          b_ph ^= 1;
        }
        if (t >= sh.ns && !(ok = mbar_wait(bar(BAR_BE + bs), b_ph, abort_flag))) break;
        const int nh = it.nh();
        mbar_expect_tx(bar(BAR_BF + bs), (u32)(sh.natoms * nh * sh.a_atom_bytes));
        const int y = (int)(TC_T * (it.blk + it.J));
        for (int a = 0; a < sh.natoms; ++a)
          for (int h = 0; h < nh; ++h)
            tma_load_2d(smem_u32(sB + bs * sh.b_bytes + a * sh.b_atom_bytes + h * sh.a_atom_bytes), &tmB, a * 64,
                        y + TC_T * h, bar(BAR_BF + bs));
      }
      if (!ok) {
        set_status(status, PH_ERR_ITER_LIMIT);
        // drain: every load issued completes before the CTA exits
        for (i64 k = (t > sh.ns ? t - sh.ns : 0); k < t; ++k)
          mbar_wait(bar(BAR_BF + (int)(k % sh.ns)), (u32)(k / sh.ns) & 1, nullptr);
        for (int k = (u - sh.na + 1 > 0 ? u - sh.na + 1 : 0); k <= u; ++k)
          mbar_wait(bar(BAR_AF + k % sh.na), (u32)(k / sh.na) & 1, nullptr);
      }
    }
    __syncwarp();
  } else if (T > 0 && warp == TC_MMA_WARP) {
    if (lane == 0) {
      const u32 idesc1 = umma_idesc_bf16_f32(TC_T, TC_T), idesc2 = umma_idesc_bf16_f32(TC_T, 2 * TC_T);
      const int spa = sh.box_k / 16;  // K slices per swizzle row
      const u64 a_step = (u64)(sh.a_atom_bytes >> 4), b_step = (u64)(sh.b_atom_bytes >> 4);
      ItemIt it{segs, blk_off, item_off, nsegs, sh.nb};
      it.start(b0);
      // as for the producer; the full-barrier phase of use v has parity v & 1
      int as = -1, bs = -1;
      u32 a_ph = 1, b_ph = 1;
      bool new_a = true;
      i64 done = 0;
      bool ok = true;
      for (i64 t = 0; t < T; ++t) {
        if (t) {
          new_a = it.row_end();
          it.next();
        }
        if (new_a) {
          if (++as == sh.na) {
            as = 0;
            a_ph ^= 1;
          }
          if (!(ok = mbar_wait(bar(BAR_AF + as), a_ph ^ 1, abort_flag))) break;
        }
        const bool last_a = (t + 1 == T) || it.row_end();
        if (++bs == sh.ns) {
          bs = 0;
          b_ph ^= 1;
        }
        if (!(ok = mbar_wait(bar(BAR_BF + bs), b_ph ^ 1, abort_flag))) break;
        const int ts = (int)(t & 1);
        if (t >= 2 && !(ok = mbar_wait(bar(BAR_TE + ts), (u32)((t >> 1) - 1) & 1, abort_flag))) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int ks = (it.sg.d + TC_AUG + 15) / 16;
        const u32 idesc = it.nh() == 2 ? idesc2 : idesc1;
        const u64 da0 = umma_desc(smem_u32(sA + as * sh.a_bytes), sh.layout, sh.sbo);
        const u64 db0 = umma_desc(smem_u32(sB + bs * sh.b_bytes), sh.layout, sh.sbo);
        // K slice s sits in swizzle atom s / spa at 32-byte step s % spa, kept
        // incrementally: a division per MMA on this one thread cost more than
        // the MMA itself
        u64 da = da0, db = db0;
        for (int s = 0, sub = 0; s < ks; ++s) {
          umma_bf16(tmem + (u32)ts * stage_cols, da, db, idesc, s > 0 ? 1u : 0u);
          if (++sub == spa) {
            sub = 0;
            da += a_step - (u64)(2 * (spa - 1));
            db += b_step - (u64)(2 * (spa - 1));
          } else {
            da += 2;
            db += 2;
          }
        }
        umma_commit(bar(BAR_BE + bs));
        umma_commit(bar(BAR_TF + ts));
        if (last_a) umma_commit(bar(BAR_AE + as));
        done = t + 1;
      }
      if (!ok) {
        set_status(status, PH_ERR_ITER_LIMIT);
        // drain: the accumulators of the last MMAs issued
        for (i64 k = (done > 2 ? done - 2 : 0); k < done; ++k)
          mbar_wait(bar(BAR_TF + (int)(k & 1)), (u32)(k / 2) & 1, nullptr);
      }
    }
    __syncwarp();
  } else if (T > 0 && warp < TC_EPI_WARPS) {
    // warpgroup g takes the items t = g, g + 2, ... (TMEM stage g). Candidates
    // are queued as cloud-local pairs across items and recomputed 32 at a
    // time (when the queue fills, the cloud changes, or the range ends), so the
    // latency of the exact chain's loads is paid once per 32 candidates.
    const int q4 = warp & 3, g = warp >> 2;
    const int row = q4 * 32 + lane;
    const u32 lt = lanemask_lt();
    uint2* queue = qbase + warp * TC_QCAP;
    unsigned long long n_cand = 0, n_forced = 0;
    int cnt = 0;
    ph_cloud_seg qs{};  // cloud of the queued candidates
    float sqthr = 0.0f;  // sqrt of the widened threshold of that cloud, rounded up
    auto flush = [&]() {
      flush_queue(queue, cnt, qs, pts_all, oi, oj, od, cap, count);
      n_cand += (unsigned long long)cnt;
      cnt = 0;
    };
    ItemIt it{segs, blk_off, item_off, nsegs, sh.nb};
    it.start(b0);
    if (g == 1 && T > 1) it.next();
    for (i64 t = g; t < T; t += 2) {
      const ph_cloud_seg& sg = it.sg;
      const bool new_cloud = sg.pt_off != qs.pt_off || sg.vbase != qs.vbase || t == g;
      if (cnt && new_cloud) flush();
      qs = sg;
      const int nh = it.nh();
      const i64 i0 = it.I * TC_T, j0 = it.J * TC_T;
      // widened thresholds of the item's column blocks, computed while the MMAs
      // run: (sqrt(thr') + r_I + r_J)^2 (1 + 2^-20) + 2^-96 with every FP32
      // operation rounded up (an upper bound of that value; the square root,
      // in FP64, once per cloud)
      if (new_cloud) sqthr = __double2float_ru(sqrt((double)sg.thr_sq * thr_scale));
      const float rt = __fadd_ru(sqthr, blkrad[it.blk + it.I]);
      float base[2];
      bool force[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float radius = __fadd_ru(rt, h < nh ? blkrad[it.blk + it.J + h] : 0.0f);
        const float b = __fadd_ru(__fmul_ru(__fmul_ru(radius, radius), 1.0f + 0x1p-20f), 0x1p-96f);
        force[h] = !(b < 3.0e38f);
        base[h] = force[h] ? 0.0f : b;
      }
      // one compare per pair into a lane mask; the set bits are queued one per
      // lane per round (a round per candidate in the densest lane)
      // the smallest of a lane's 32 values (a min tree)
      auto vmin = [](const u32 (&v)[32]) {
        float m16[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) m16[k] = fminf(__uint_as_float(v[k]), __uint_as_float(v[k + 16]));
#pragma unroll
        for (int w = 8; w > 0; w >>= 1)
#pragma unroll
          for (int k = 0; k < w; ++k) m16[k] = fminf(m16[k], m16[k + w]);
        return m16[0];
      };
      // the candidates among a lane's 32 values, queued
      auto screen = [&](const u32 (&v)[32], int c0, float bs_) {
        u32 mask = 0;
#pragma unroll
        for (int k = 0; k < 32; ++k) mask |= (__uint_as_float(v[k]) < bs_ ? 1u : 0u) << k;
#pragma unroll 1
        while (__any_sync(FULL, mask != 0)) {
          const bool has = mask != 0;
          const u32 m = __ballot_sync(FULL, has);
          if (cnt + 32 > TC_QCAP) flush();
          if (has) {
            const int k = __ffs(mask) - 1;
            queue[cnt + __popc(m & lt)] = make_uint2((u32)(i0 + row), (u32)(j0 + c0 + k));
            mask &= mask - 1;
          }
          cnt += __popc(m);
        }
      };
      int okw = 1;
      if (lane == 0) okw = mbar_wait(bar(BAR_TF + g), (u32)(t >> 1) & 1, abort_flag) ? 1 : 0;
      okw = __shfl_sync(FULL, okw, 0);
      if (!okw) {
        if (lane == 0) set_status(status, PH_ERR_ITER_LIMIT);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const u32 taddr = tmem + (u32)g * stage_cols + ((u32)(q4 * 32) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < TC_T * nh; c0 += 64) {
        const int h = c0 >> 7;
        if (force[h]) continue;
        u32 v0[32], v1[32];
        tmem_ld32_issue(taddr + (u32)c0, v0);
        tmem_ld32_issue(taddr + (u32)(c0 + 32), v1);
        tmem_ld_wait();
        // both min trees before one vote: independent chains side by side and
        // one branch per 64 columns (almost always: no candidate)
        const float mn = fminf(vmin(v0), vmin(v1));
        if (!__any_sync(FULL, mn < base[h])) continue;
        screen(v0, c0, base[h]);
        screen(v1, c0 + 32, base[h]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(BAR_TE + g));
      for (int h = 0; h < nh; ++h) {
        if (!force[h]) continue;
        // no screen for this column block: every pair of the warp's rows exactly
        n_forced += 32 * TC_T;
        const float* P = pts_all + sg.pt_off;
        const i64 gi = i0 + row;
        for (int col = 0; col < TC_T; ++col) {
          const i64 gj = j0 + h * TC_T + col;
          bool emit = false;
          float acc = 0.0f;
          if (gi < gj && gj < sg.n) {
            acc = exact_dsq(P + gi * sg.d, P + gj * sg.d, sg.d);
            emit = acc < sg.thr_sq;
          }
          emit_warp(emit, sg.vbase + gi, sg.vbase + gj, acc, lane, oi, oj, od, cap, count);
        }
      }
      if (t + 2 < T) {
        it.next();
        it.next();
      }
    }
    if (cnt) flush();
    if (stats && lane == 0) {
      atomicAdd(&st_sh[0], n_cand);
      atomicAdd(&st_sh[1], n_forced);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == TC_MMA_WARP) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * stage_cols));
  }
  if (stats && threadIdx.x == 0) {
    if (st_sh[0]) atomicAdd(&stats[0], st_sh[0]);
    if (st_sh[1]) atomicAdd(&stats[1], st_sh[1]);
  }
}

}  // namespace
}  // namespace ph

using namespace ph;

namespace {

struct TcPlan {
  TcShape sh;
  size_t smem;
};

TcPlan plan_for(int max_d) {
  TcPlan p;
  TcShape& s = p.sh;
  s.kq = tc_kq(max_d);
  s.box_k = std::min(s.kq, 64);
  s.natoms = s.kq / s.box_k;
  s.row_bytes = s.box_k * 2;
  s.a_atom_bytes = TC_T * s.row_bytes;
  s.a_bytes = s.natoms * s.a_atom_bytes;
  s.layout = s.box_k == 16 ? 6u : s.box_k == 32 ? 4u : 2u;
  s.sbo = (u32)(8 * s.row_bytes) >> 4;
  const size_t queues = (size_t)TC_EPI_WARPS * TC_QCAP * sizeof(uint2);
  const size_t budget = 227 * 1024 - 1024 - queues;
  // widest items (N = 256) whose rings still hold two B stages
  for (int nb = 2; nb >= 1; --nb) {
    s.nb = nb;
    s.b_atom_bytes = nb * s.a_atom_bytes;
    s.b_bytes = s.natoms * s.b_atom_bytes;
    for (int na = 2; na >= 1; --na) {
      if (budget < (size_t)na * s.a_bytes) continue;
      const int ns = (int)((budget - (size_t)na * s.a_bytes) / s.b_bytes);
      if (ns >= 2) {
        s.na = na;
        s.ns = std::min(ns, TC_MAX_STAGES);
        // at least 120 KB so that one CTA (and its TMEM columns) holds an SM
        p.smem = std::max<size_t>(1024 + (size_t)s.na * s.a_bytes + (size_t)s.ns * s.b_bytes + queues, 120 * 1024);
        return p;
      }
    }
  }
  s.nb = 0;  // unreachable for kq <= 256
  p.smem = 0;
  return p;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// 2-D BF16 map over rows x kq, box = 128 rows x box_k columns, swizzled like the UMMA layout
bool make_map(CUtensorMap* m, void* base, i64 rows, const TcShape& s) {
  auto enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)s.kq, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)s.kq * 2};
  const cuuint32_t box[2] = {(cuuint32_t)s.box_k, (cuuint32_t)TC_T};
  const cuuint32_t es[2] = {1, 1};
  const CUtensorMapSwizzle sw = s.box_k == 16   ? CU_TENSOR_MAP_SWIZZLE_32B
                                : s.box_k == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                : CU_TENSOR_MAP_SWIZZLE_128B;
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

extern "C" size_t ph_edges_screened_workspace_bytes(int64_t N, int32_t nsegs, int32_t max_d) {
  if (N < 0 || nsegs < 1 || max_d < 1 || max_d > TC_MAXK - TC_AUG) return 0;
  const TcPlan p = plan_for(max_d);
  const size_t rows = (size_t)N + (size_t)TC_T * nsegs;  // padded rows (each cloud to a multiple of 128)
  return 2 * Carve::need(rows * p.sh.kq * sizeof(__nv_bfloat16)) + Carve::need(rows / TC_T * sizeof(float) + 4) +
         Carve::need((size_t)nsegs * TC_MAXK * sizeof(double)) + Carve::need((size_t)(nsegs + 1) * sizeof(i64));
}

extern "C" int ph_batch_edges_enumerate_screened(const float* pts, const ph_cloud_seg* segs, int32_t nsegs,
                                                 int64_t ntiles, int32_t max_d, int64_t N, const int64_t* blk_off,
                                                 int64_t nblocks, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                                 int64_t capacity, unsigned long long* d_count, int* d_status,
                                                 unsigned long long* d_stats, void* workspace,
                                                 size_t workspace_bytes, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (nsegs < 1 || ntiles < 0 || max_d < 1 || max_d > TC_MAXK - TC_AUG || N < 0 || capacity < 0 || !d_count ||
      !segs || !blk_off || nblocks < 0 || nblocks > (N + (i64)TC_T * nsegs) / TC_T) {
    record_message("ph_batch_edges_enumerate_screened: invalid argument (d must be in [1, 252])");
    return PH_ERR_ARG;
  }
  if (ntiles >= (int64_t(1) << 31) || nblocks * TC_T >= (int64_t(1) << 31)) return PH_ERR_OVERFLOW;
  const TcPlan p = plan_for(max_d);
  const i64 rows = std::max<i64>(nblocks, 1) * TC_T;
  Carve c(workspace, workspace_bytes);
  __nv_bfloat16* YA = c.take<__nv_bfloat16>(rows * p.sh.kq);
  __nv_bfloat16* YB = c.take<__nv_bfloat16>(rows * p.sh.kq);
  float* blkrad = c.take<float>(std::max<i64>(nblocks, 1));
  double* sum = c.take<double>((i64)nsegs * TC_MAXK);
  i64* item_off = c.take<i64>((i64)nsegs + 1);
  if (!YA || !YB || !blkrad || !sum || !item_off || p.sh.nb == 0) {
    record_message("ph_batch_edges_enumerate_screened: workspace too small");
    return PH_ERR_ARG;
  }
  if (ntiles == 0 || N == 0 || nblocks == 0) {
    ph::zero_async(d_count, sizeof(unsigned long long), s);
    PH_CHECK_LAUNCH();
    return PH_OK;
  }
  CUtensorMap tmA, tmB;
  if (!make_map(&tmA, YA, rows, p.sh) || !make_map(&tmB, YB, rows, p.sh)) {
    record_message("ph_batch_edges_enumerate_screened: tensor map encoding failed");
    return PH_ERR_CUDA;
  }
  if (ph::allow_dynamic_smem((const void*)k_tc_edges) != cudaSuccess) {
    PH_CHECK_LAUNCH();
    return PH_ERR_CUDA;
  }
  const int sms = ph::device_sms();
  const int occ = ph::occupancy((const void*)k_tc_edges, TC_THREADS, p.smem);
  if (occ != 1) {
    record_message("ph_batch_edges_enumerate_screened: expected one CTA per SM for the TMEM budget");
    return PH_ERR_CUDA;
  }
  ph::zero_async(sum, sizeof(double) * nsegs * TC_MAXK, s, d_count, sizeof(unsigned long long));
  const double kappa = std::max(0x1p-11, (double)p.sh.kq * 0x1p-18);
  ph::count_launch();
  ph::launch_pdl(k_tc_mean, dim3((unsigned)nblocks), dim3(256), 0, s, pts, segs, nsegs, blk_off, sum);
  ph::count_launch();
  ph::launch_pdl(k_tc_points, dim3((unsigned)nblocks), dim3(TC_T), 0, s, pts, segs, nsegs, blk_off, sum, p.sh.kq, kappa, YA, YB, blkrad);
  ph::count_launch();
  ph::launch_pdl(k_tc_items, dim3(1), dim3(1024), 0, s, segs, nsegs, p.sh.nb, item_off);
  const double thr_scale = 1.0 + (double)(max_d + 3) * 0x1p-24;
  // persistent: one CTA per SM, each a contiguous range of the items (counted on the device)
  const int grid = (int)std::min<i64>(ntiles, (i64)sms);
  ph::count_launch();
  ph::launch_pdl(k_tc_edges, dim3(grid), dim3(TC_THREADS), p.smem, s, tmA, tmB, pts, segs, nsegs, blk_off, item_off, blkrad, p.sh,
                                              thr_scale, out_i, out_j, out_dsq, capacity, d_count, d_status, d_stats);
  PH_CHECK_LAUNCH();
  return PH_OK;
}
