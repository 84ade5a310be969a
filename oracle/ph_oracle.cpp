// CPU oracle for exact Vietoris-Rips persistent homology (H0/H1/H2 over Z/2).
//
// TEST INFRASTRUCTURE ONLY. This file restates, step by step, the algorithm
// of the reference implementation (ot-triton-lab/flash-ph) so that the CUDA
// path can be checked against it. It is never the thing measured or shipped:
// only the tests, the smoke check and the CPU-baseline leg of bench.py load
// it. Every function cites the reference file:line it follows.
//
// Build: make -C oracle   (produces oracle/_build/libph_oracle.so)
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>
#include <atomic>
#include <thread>

namespace {

using i32 = int32_t;
using i64 = int64_t;
using u32 = uint32_t;
using u64 = uint64_t;

struct Result {
  // sorted filtration (rips.py:15-27)
  std::vector<i32> edge_i, edge_j;
  std::vector<float> edge_dsq;
  // H0 (boruvka.py, persistence.py:169-192)
  std::vector<i64> mst_idx;
  i64 n_components = 0;
  std::vector<float> h0;
  // H1 (reduce_h1_gpu.py:438-604)
  i64 T = 0, cofacet_nnz = 0, n_apparent = 0, residual = 0;
  i64 xor_ops = 0, xor_max = 0, xor_elems = 0;  // reduction work statistics
  i64 crit_path = 0;  // H1: longest chain of dependent additions (each waits for the column it adds)
  i64 col_max = 0;    // H1: largest working column (entries) met during the reduction
  std::vector<i32> tri_max_rank_sorted;
  std::vector<i32> ap_births, ap_deaths, res_births, res_deaths, ess_births;
  std::vector<i32> h1_all_pivots;
  std::vector<float> h1;
  // H2 (assembled from triangle_kernel.py:402, cohomology_general.py:32)
  i64 Q = 0;
  std::vector<float> h2;
  std::vector<i32> h2_births, h2_deaths, h2_ess;
  // edge collapse (oracle_run_collapsed): edges of the full filtration, edges
  // dropped, edges inserted later than their own time
  i64 E_full = 0, collapse_removed = 0, collapse_delayed = 0, collapse_rounds = 0;
  std::vector<i64> slot_seq, slot_rounds;  // oracle_collapse_slots
  std::string error;
};

inline u32 fbits(float f) {
  u32 u;
  std::memcpy(&u, &f, 4);
  return u;
}

// --- edge enumeration: kernels/edge_kernel.py:23-149,152-224 -------------
// Tiles of B=32 points, programs (I, J) with I <= J in row-major order of the
// flattened nb x nb grid (prefix at edge_kernel.py:208-210); inside a tile the
// emitted order is row-major over (source offset, target offset)
// (edge_kernel.py:134-149). dist^2 is accumulated over k = 0..d-1 in order
// (edge_kernel.py:111-123): fused (one rounding per step, fmaf) or as a
// separate multiply and add (this file is compiled with -ffp-contract=off).
template <bool FUSED>
static void tile_row(const float* pts, i64 n, int d, float thr_sq, i64 I, i64 nb,
                     std::vector<i32>& vi, std::vector<i32>& vj, std::vector<float>& vd) {
  const i64 B = 32;
  for (i64 J = I; J < nb; ++J) {
    for (i64 a = 0; a < B; ++a) {
      const i64 i = I * B + a;
      if (i >= n) break;
      const float* x = pts + i * d;
      for (i64 b = (I == J ? a + 1 : 0); b < B; ++b) {
        const i64 j = J * B + b;
        if (j >= n) break;
        const float* y = pts + j * d;
        float acc = 0.0f;
        for (int k = 0; k < d; ++k) {
          const float df = x[k] - y[k];
          if (FUSED) acc = __builtin_fmaf(df, df, acc);
          else acc = acc + df * df;
        }
        if (acc < thr_sq) {
          vi.push_back((i32)i);
          vj.push_back((i32)j);
          vd.push_back(acc);
        }
      }
    }
  }
}
__attribute__((target("fma"))) static void tile_row_fma_hw(
    const float* pts, i64 n, int d, float thr_sq, i64 I, i64 nb,
    std::vector<i32>& vi, std::vector<i32>& vj, std::vector<float>& vd) {
  tile_row<true>(pts, n, d, thr_sq, I, nb, vi, vj, vd);
}

void enumerate_edges(const float* pts, i64 n, int d, float thr_sq, int fused,
                     int nthreads, std::vector<i32>& oi, std::vector<i32>& oj,
                     std::vector<float>& odsq) {
  const i64 B = 32;
  const i64 nb = (n + B - 1) / B;
  const bool hw_fma = __builtin_cpu_supports("fma");
  std::vector<std::vector<i32>> ri(nb), rj(nb);
  std::vector<std::vector<float>> rd(nb);
  // Tile rows are independent; threads take them dynamically (largest rows
  // first) and the per-row lists are concatenated in row order afterwards, so
  // the emitted order does not depend on the thread count.
  std::atomic<i64> next{0};
  auto worker = [&]() {
    for (;;) {
      const i64 I = next.fetch_add(1);
      if (I >= nb) break;
      if (!fused) tile_row<false>(pts, n, d, thr_sq, I, nb, ri[I], rj[I], rd[I]);
      else if (hw_fma) tile_row_fma_hw(pts, n, d, thr_sq, I, nb, ri[I], rj[I], rd[I]);
      else tile_row<true>(pts, n, d, thr_sq, I, nb, ri[I], rj[I], rd[I]);
    }
  };
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nt > nb) nt = (int)std::max<i64>(1, nb);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  for (i64 I = 0; I < nb; ++I) {
    oi.insert(oi.end(), ri[I].begin(), ri[I].end());
    oj.insert(oj.end(), rj[I].begin(), rj[I].end());
    odsq.insert(odsq.end(), rd[I].begin(), rd[I].end());
  }
}

// --- filtration sort: rips.py:30-50,188-202 --------------------------------
// key = (float bits of dist^2) << 32 | (j(j-1)/2 + i) & 0xFFFFFFFF, stable.
void sort_edges(std::vector<i32>& ei, std::vector<i32>& ej, std::vector<float>& ed) {
  const size_t E = ei.size();
  std::vector<u64> key(E);
  for (size_t e = 0; e < E; ++e) {
    u64 j = (u64)ej[e], i = (u64)ei[e];
    u64 colex = j * (j - 1) / 2 + i;
    key[e] = ((u64)fbits(ed[e]) << 32) | (colex & 0xFFFFFFFFull);
  }
  std::vector<i64> perm(E);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](i64 a, i64 b) { return key[a] < key[b]; });
  std::vector<i32> a(E), b(E);
  std::vector<float> c(E);
  for (size_t k = 0; k < E; ++k) {
    a[k] = ei[perm[k]];
    b[k] = ej[perm[k]];
    c[k] = ed[perm[k]];
  }
  ei.swap(a);
  ej.swap(b);
  ed.swap(c);
}

// --- vertex CSR: rips.py:53-95 (rows sorted by neighbour index) -----------
struct CSR {
  std::vector<i32> ptr, idx, rank;
};
CSR vertex_csr(const std::vector<i32>& ei, const std::vector<i32>& ej, i64 n) {
  CSR g;
  const i64 E = (i64)ei.size();
  g.ptr.assign(n + 1, 0);
  for (i64 e = 0; e < E; ++e) {
    g.ptr[ei[e] + 1]++;
    g.ptr[ej[e] + 1]++;
  }
  for (i64 v = 0; v < n; ++v) g.ptr[v + 1] += g.ptr[v];
  g.idx.resize(2 * E);
  g.rank.resize(2 * E);
  std::vector<i32> fill(g.ptr.begin(), g.ptr.end() - 1);
  for (i64 e = 0; e < E; ++e) {
    int p = fill[ei[e]]++;
    g.idx[p] = ej[e];
    g.rank[p] = (i32)e;
    p = fill[ej[e]]++;
    g.idx[p] = ei[e];
    g.rank[p] = (i32)e;
  }
  std::vector<std::pair<i32, i32>> tmp;
  for (i64 v = 0; v < n; ++v) {
    tmp.clear();
    for (int p = g.ptr[v]; p < g.ptr[v + 1]; ++p) tmp.emplace_back(g.idx[p], g.rank[p]);
    std::sort(tmp.begin(), tmp.end());
    for (size_t k = 0; k < tmp.size(); ++k) {
      g.idx[g.ptr[v] + k] = tmp[k].first;
      g.rank[g.ptr[v] + k] = tmp[k].second;
    }
  }
  return g;
}

// --- Boruvka: boruvka.py:17-113, round for round ---------------------------
void boruvka(const std::vector<i32>& ei, const std::vector<i32>& ej, i64 n,
             std::vector<i64>& mst, i64& ncomp) {
  const i64 E = (i64)ei.size();
  std::vector<i64> comp(n);
  std::iota(comp.begin(), comp.end(), 0);
  std::vector<char> in_mst(E, 0);
  auto flatten = [&]() {
    std::vector<i64> nc(n);
    for (int it = 0; it < 64; ++it) {
      bool same = true;
      for (i64 v = 0; v < n; ++v) {
        nc[v] = comp[comp[v]];
        if (nc[v] != comp[v]) same = false;
      }
      if (same) break;
      comp.swap(nc);
    }
  };
  const int max_iters = (int)std::ceil(std::log2((double)std::max<i64>(n, 2))) + 2;
  const i64 SENT = INT64_MAX;
  std::vector<i64> min_key(n);
  std::vector<char> seen(n);
  for (int r = 0; r < max_iters; ++r) {
    flatten();
    std::fill(seen.begin(), seen.end(), 0);
    i64 K = 0;
    for (i64 v = 0; v < n; ++v)
      if (!seen[comp[v]]) {
        seen[comp[v]] = 1;
        ++K;
      }
    if (K == 1) break;
    std::fill(min_key.begin(), min_key.end(), SENT);
    bool any = false;
    for (i64 e = 0; e < E; ++e) {
      i64 cu = comp[ei[e]], cv = comp[ej[e]];
      if (cu == cv) continue;
      any = true;
      min_key[cu] = std::min(min_key[cu], e);
      min_key[cv] = std::min(min_key[cv], e);
    }
    if (!any) break;
    std::vector<i64> sel;
    for (i64 c = 0; c < n; ++c)
      if (min_key[c] < SENT) sel.push_back(min_key[c]);
    std::sort(sel.begin(), sel.end());
    sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
    std::vector<std::pair<i64, i64>> hooks;
    for (i64 e : sel) {
      in_mst[e] = 1;
      i64 su = comp[ei[e]], sv = comp[ej[e]];
      hooks.emplace_back(std::max(su, sv), std::min(su, sv));
    }
    for (auto& h : hooks) comp[h.first] = std::min(comp[h.first], h.second);
  }
  flatten();
  mst.clear();
  for (i64 e = 0; e < E; ++e)
    if (in_mst[e]) mst.push_back(e);
  std::vector<char> s2(n, 0);
  ncomp = 0;
  for (i64 v = 0; v < n; ++v)
    if (!s2[comp[v]]) {
      s2[comp[v]] = 1;
      ++ncomp;
    }
}

// --- Z/2 column store used by the reducers (cohomology_general.py) ---------
// The reference keeps reduced columns in a pool addressed through an
// open-addressing hash map keyed by pivot (_numba_utils.py:14-40); a map from
// pivot to column is the same mapping.
using Col = std::vector<i32>;
void xor_into(Col& cur, const Col& other, Col& tmp) {  // _numba_utils.py:43-65
  tmp.clear();
  size_t a = 0, b = 0;
  while (a < cur.size() && b < other.size()) {
    if (cur[a] < other[b]) tmp.push_back(cur[a++]);
    else if (cur[a] > other[b]) tmp.push_back(other[b++]);
    else { ++a; ++b; }
  }
  while (a < cur.size()) tmp.push_back(cur[a++]);
  while (b < other.size()) tmp.push_back(other[b++]);
  cur.swap(tmp);
}

// Sorted-vertex colex ids (cohomology_general.py:378-415, overflow-safe tet
// form apparent_pair_h2_kernel.py:53-58).
inline i64 tri_colex(i64 a, i64 b, i64 c) { return c * (c - 1) * (c - 2) / 6 + b * (b - 1) / 2 + a; }
inline i64 tet_colex(i64 a, i64 b, i64 c, i64 d) {
  i64 hi = d * (d - 1) / 2, lo = (d - 2) * (d - 3) / 2;
  return hi * lo / 6 + c * (c - 1) * (c - 2) / 6 + b * (b - 1) / 2 + a;
}

i32 edge_rank_lookup(const CSR& g, i32 s, i32 t) {  // apparent_pair_h2_kernel.py:37-49
  int lo = g.ptr[s], hi = g.ptr[s + 1];
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (g.idx[mid] < t) lo = mid + 1;
    else if (g.idx[mid] > t) hi = mid;
    else return g.rank[mid];
  }
  return -1;
}

void stable_sort_rows_by_birth(std::vector<float>& rows) {
  const size_t K = rows.size() / 2;
  std::vector<size_t> p(K);
  std::iota(p.begin(), p.end(), 0);
  std::stable_sort(p.begin(), p.end(), [&](size_t a, size_t b) { return rows[2 * a] < rows[2 * b]; });
  std::vector<float> out(rows.size());
  for (size_t k = 0; k < K; ++k) {
    out[2 * k] = rows[2 * p[k]];
    out[2 * k + 1] = rows[2 * p[k] + 1];
  }
  rows.swap(out);
}

struct Triangles {  // triangle_kernel.py:288-399 output, plus ranks
  std::vector<i32> v0, v1, v2, mr;
  std::vector<i32> grank;      // global rank E + position in (max_rank, colex) order
  std::vector<i32> sorted_idx; // triangle index at each sorted position
};

// triangle_kernel.py:81-144 / _numba_utils.py:111-183: per edge in rank order,
// common neighbours w > v in increasing order; max_rank over the three edges.
Triangles enumerate_triangles(const std::vector<i32>& ei, const std::vector<i32>& ej, const CSR& g) {
  Triangles t;
  const i64 E = (i64)ei.size();
  for (i64 e = 0; e < E; ++e) {
    i32 u = std::min(ei[e], ej[e]), v = std::max(ei[e], ej[e]);
    int iu = g.ptr[u], iv = g.ptr[v];
    const int ue = g.ptr[u + 1], ve = g.ptr[v + 1];
    while (iu < ue && iv < ve) {
      i32 nu = g.idx[iu], nv = g.idx[iv];
      if (nu == nv) {
        if (nu > v) {
          t.v0.push_back(u);
          t.v1.push_back(v);
          t.v2.push_back(nu);
          t.mr.push_back(std::max<i32>((i32)e, std::max(g.rank[iu], g.rank[iv])));
        }
        ++iu;
        ++iv;
      } else if (nu < nv) {
        ++iu;
      } else {
        ++iv;
      }
    }
  }
  // reduce_h1_gpu.py:509-521: order by (max_rank, colex), global rank = E + pos
  const i64 T = (i64)t.v0.size();
  std::vector<i64> colex(T);
  for (i64 k = 0; k < T; ++k) colex[k] = tri_colex(t.v0[k], t.v1[k], t.v2[k]);
  t.sorted_idx.resize(T);
  std::iota(t.sorted_idx.begin(), t.sorted_idx.end(), 0);
  std::stable_sort(t.sorted_idx.begin(), t.sorted_idx.end(),
                   [&](i32 a, i32 b) { return colex[a] < colex[b]; });
  std::stable_sort(t.sorted_idx.begin(), t.sorted_idx.end(),
                   [&](i32 a, i32 b) { return t.mr[a] < t.mr[b]; });
  t.grank.resize(T);
  for (i64 p = 0; p < T; ++p) t.grank[t.sorted_idx[p]] = (i32)(E + p);
  return t;
}

// reduce_h1_gpu.py:438-604 (apparent pairs reduce_h1_gpu.py:159-223, residual
// reduction cohomology_general.py:202-371 with the pool prepopulated by the
// apparent columns, _numba_utils.py:68-104).
void h1_native(Result& R, i64 n, const CSR& g, const Triangles& tr, const std::vector<char>& mst_mask,
               const std::vector<float>& edge_filt) {
  const i64 E = (i64)R.edge_i.size();
  const i64 T = (i64)tr.v0.size();
  R.T = T;
  if (T == 0) {  // reduce_h1_gpu.py:495-502
    for (i64 e = 0; e < E; ++e)
      if (!mst_mask[e]) {
        R.h1.push_back(edge_filt[e]);
        R.h1.push_back(INFINITY);
      }
    stable_sort_rows_by_birth(R.h1);
    return;
  }
  // face ranks (reduce_h1_gpu.py:65-100) and cofacet CSR (:107-152)
  std::vector<std::vector<i32>> cof(E);
  for (i64 k = 0; k < T; ++k) {
    i32 a = tr.v0[k], b = tr.v1[k], c = tr.v2[k];
    i32 f[3] = {edge_rank_lookup(g, a, b), edge_rank_lookup(g, a, c), edge_rank_lookup(g, b, c)};
    for (int q = 0; q < 3; ++q) cof[f[q]].push_back(tr.grank[k]);
  }
  for (auto& r : cof) std::sort(r.begin(), r.end());
  for (auto& r : cof) R.cofacet_nnz += (i64)r.size();
  // rank_to_filt (reduce_h1_gpu.py:528-530)
  std::vector<float> r2f(edge_filt);
  for (i64 p = 0; p < T; ++p) r2f.push_back(edge_filt[tr.mr[tr.sorted_idx[p]]]);
  R.tri_max_rank_sorted.resize(T);
  for (i64 p = 0; p < T; ++p) R.tri_max_rank_sorted[p] = tr.mr[tr.sorted_idx[p]];
  // cof_max_face: max non-skipped face rank of each cofacet
  std::vector<i32> cmf(E + T, -1);
  for (i64 e = 0; e < E; ++e) {
    if (mst_mask[e]) continue;
    for (i32 t : cof[e]) cmf[t] = std::max(cmf[t], (i32)e);
  }
  std::vector<char> is_app(E, 0);
  std::map<i32, Col> table;
  std::map<i32, i64> done_at;  // pivot -> step at which its column became final
  for (i64 e = 0; e < E; ++e) {
    if (cof[e].empty() || mst_mask[e]) continue;
    if (cmf[cof[e][0]] == (i32)e) {
      is_app[e] = 1;
      R.n_apparent++;
      i32 piv = cof[e][0];
      R.h1_all_pivots.push_back(piv);
      if (r2f[piv] > r2f[e]) {
        R.ap_births.push_back((i32)e);
        R.ap_deaths.push_back(piv);
      }
      table[piv] = cof[e];
    }
  }
  Col cur, tmp;
  for (i64 e = E - 1; e >= 0; --e) {
    if (mst_mask[e] || is_app[e]) continue;
    R.residual++;
    if (cof[e].empty()) {
      R.ess_births.push_back((i32)e);
      continue;
    }
    cur = cof[e];
    i64 ops = 0, step = 0;
    while (!cur.empty()) {
      auto it = table.find(cur[0]);
      if (it == table.end()) break;
      auto dt = done_at.find(cur[0]);
      step = std::max(step, dt == done_at.end() ? (i64)0 : dt->second) + 1;
      R.xor_elems += (i64)(cur.size() + it->second.size());
      xor_into(cur, it->second, tmp);
      R.col_max = std::max<i64>(R.col_max, (i64)cur.size());
      ++ops;
    }
    R.crit_path = std::max(R.crit_path, step);
    R.xor_ops += ops;
    R.xor_max = std::max(R.xor_max, ops);
    if (!cur.empty()) {
      i32 piv = cur[0];
      R.h1_all_pivots.push_back(piv);
      table[piv] = cur;
      done_at[piv] = step;
      if (r2f[piv] > r2f[e]) {
        R.res_births.push_back((i32)e);
        R.res_deaths.push_back(piv);
      }
    } else {
      R.ess_births.push_back((i32)e);
    }
  }
  // assembly (reduce_h1_gpu.py:574-604)
  for (size_t k = 0; k < R.ap_births.size(); ++k) {
    R.h1.push_back(r2f[R.ap_births[k]]);
    R.h1.push_back(r2f[R.ap_deaths[k]]);
  }
  for (size_t k = 0; k < R.res_births.size(); ++k) {
    R.h1.push_back(r2f[R.res_births[k]]);
    R.h1.push_back(r2f[R.res_deaths[k]]);
  }
  for (i32 e : R.ess_births) {
    R.h1.push_back(r2f[e]);
    R.h1.push_back(INFINITY);
  }
  stable_sort_rows_by_birth(R.h1);
}

// H2: tetrahedra (triangle_kernel.py:152-270 / _numba_utils.py:186-284),
// ordered by (max_rank, colex) (apparent_pair_h2_kernel.py:117-121), columns
// are the triangles in their global order with the H1 pivots cleared, reduced
// by the general cohomology reducer (cohomology_general.py:32-199).
void h2_blocks(Result& R, const CSR& g, const Triangles& tr, const std::vector<float>& edge_filt) {
  const i64 E = (i64)R.edge_i.size();
  const i64 T = (i64)tr.v0.size();
  std::vector<i32> q0, q1, q2, q3, qmr;
  for (i64 k = 0; k < T; ++k) {
    i32 a = tr.v0[k], b = tr.v1[k], c = tr.v2[k];
    int ia = g.ptr[a], ib = g.ptr[b], ic = g.ptr[c];
    const int ae = g.ptr[a + 1], be = g.ptr[b + 1], ce = g.ptr[c + 1];
    while (ia < ae && ib < be && ic < ce) {
      i32 na = g.idx[ia], nb = g.idx[ib], nc = g.idx[ic];
      i32 mx = std::max(na, std::max(nb, nc));
      if (na == nb && nb == nc) {
        if (na > c) {
          q0.push_back(a);
          q1.push_back(b);
          q2.push_back(c);
          q3.push_back(na);
          qmr.push_back(std::max(tr.mr[k], std::max(g.rank[ia], std::max(g.rank[ib], g.rank[ic]))));
        }
        ++ia;
        ++ib;
        ++ic;
      } else {
        if (na < mx) ++ia;
        if (nb < mx) ++ib;
        if (nc < mx) ++ic;
      }
    }
  }
  const i64 Q = (i64)q0.size();
  R.Q = Q;
  std::vector<i64> colex(Q);
  for (i64 k = 0; k < Q; ++k) colex[k] = tet_colex(q0[k], q1[k], q2[k], q3[k]);
  std::vector<i32> ord(Q);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](i32 a, i32 b) {
    return qmr[a] != qmr[b] ? qmr[a] < qmr[b] : colex[a] < colex[b];
  });
  std::vector<i32> qrank(Q);
  for (i64 p = 0; p < Q; ++p) qrank[ord[p]] = (i32)(E + T + p);
  // packed triangle key v0 + v1<<16 + v2<<32 (n < 65536)
  std::unordered_map<u64, i32> tkey;
  tkey.reserve(T * 2);
  auto pack = [](u64 a, u64 b, u64 c) { return a | (b << 16) | (c << 32); };
  std::vector<i32> tpos(T);  // triangle index -> local column index (global - E)
  for (i64 k = 0; k < T; ++k) {
    tkey[pack(tr.v0[k], tr.v1[k], tr.v2[k])] = (i32)k;
    tpos[k] = tr.grank[k] - (i32)E;
  }
  std::vector<std::vector<i32>> cof(T);  // by local triangle column index
  for (i64 k = 0; k < Q; ++k) {
    u64 a = q0[k], b = q1[k], c = q2[k], d = q3[k];
    u64 f[4] = {pack(a, b, c), pack(a, b, d), pack(a, c, d), pack(b, c, d)};
    for (int z = 0; z < 4; ++z) cof[tpos[tkey.at(f[z])]].push_back(qrank[k]);
  }
  for (auto& r : cof) std::sort(r.begin(), r.end());
  // rank -> filtration value over edges, triangles, tetrahedra
  std::vector<float> r2f(edge_filt);
  for (i64 p = 0; p < T; ++p) r2f.push_back(edge_filt[tr.mr[tr.sorted_idx[p]]]);
  for (i64 p = 0; p < Q; ++p) r2f.push_back(edge_filt[qmr[ord[p]]]);
  // clearing: triangles that are H1 pivots are skipped
  std::vector<char> skip(T, 0);
  for (i32 piv : R.h1_all_pivots) skip[piv - E] = 1;
  std::vector<i32> cmf(E + T + Q, -1);
  for (i64 c = 0; c < T; ++c) {
    if (skip[c]) continue;
    for (i32 t : cof[c]) cmf[t] = std::max(cmf[t], (i32)(E + c));
  }
  std::map<i32, Col> table;
  Col cur, tmp;
  for (i64 c = T - 1; c >= 0; --c) {
    if (skip[c]) continue;
    const i32 r = (i32)(E + c);
    if (cof[c].empty()) {
      R.h2_ess.push_back(r);
      continue;
    }
    i32 young = cof[c][0];
    if (cmf[young] == r) {
      table[young] = cof[c];
      if (r2f[young] > r2f[r]) {
        R.h2_births.push_back(r);
        R.h2_deaths.push_back(young);
      }
      continue;
    }
    cur = cof[c];
    while (!cur.empty()) {
      auto it = table.find(cur[0]);
      if (it == table.end()) break;
      xor_into(cur, it->second, tmp);
    }
    if (!cur.empty()) {
      table[cur[0]] = cur;
      if (r2f[cur[0]] > r2f[r]) {
        R.h2_births.push_back(r);
        R.h2_deaths.push_back(cur[0]);
      }
    } else {
      R.h2_ess.push_back(r);
    }
  }
  for (size_t k = 0; k < R.h2_births.size(); ++k) {
    R.h2.push_back(r2f[R.h2_births[k]]);
    R.h2.push_back(r2f[R.h2_deaths[k]]);
  }
  for (i32 r : R.h2_ess) {
    R.h2.push_back(r2f[r]);
    R.h2.push_back(INFINITY);
  }
  stable_sort_rows_by_birth(R.h2);
}

}  // namespace

// --- Edge collapse of the flag filtration -------------------------------
// The reference computes H2 with giotto-ph's ripser_parallel(...,
// collapse_edges=True) (persistence.py:48-51): the flag filtration is first
// shrunk by edge collapses, which leave every persistence diagram unchanged.
// giotto-ph (PyPI giotto-ph, unpinned in the reference's pyproject.toml) is not
// part of the reference tree; this restates the published criterion (Boissonnat
// and Pritam, "Edge collapse and persistence of flag complexes", SoCG 2020)
// rather than that library's code. An edge uv is dominated in a graph when a
// vertex w adjacent to u and v is adjacent to every other common neighbour of
// u and v; removing a dominated edge is a strong collapse of the flag complex,
// so the smaller complex includes into the larger by a homotopy equivalence.
// Edges are taken from the last to the first. Each is inserted at the first
// time (original edge index) at which it is not dominated in the graph of that
// time -- earlier edges at their own times, later ones at the times already
// chosen -- and dropped if it stays dominated to the end. Each such move keeps
// the graph of every time the old graph minus an edge dominated in it, so the
// persistence modules stay isomorphic through the inclusions and the diagrams,
// read by filtration value, are unchanged. Test infrastructure: it shows that
// a collapsed and an uncollapsed filtration give the same diagrams.
//
// slot[e] = the time from which edge e is present after the collapse (e itself
// when unchanged), -1 when dropped. Dense n x n table: small inputs only.
bool collapse_edges(i64 n, const std::vector<i32>& ei, const std::vector<i32>& ej, std::vector<i64>& slot,
                    i64& removed, i64& delayed) {
  const i64 E = (i64)ei.size();
  const i32 NONE = INT32_MAX;
  if (n > 4096) return false;
  std::vector<i32> at((size_t)(n * n), NONE);  // at[a * n + b]: time from which edge ab is present
  for (i64 e = 0; e < E; ++e) at[(size_t)(ei[e] * n + ej[e])] = at[(size_t)(ej[e] * n + ei[e])] = (i32)e;
  slot.assign(E, 0);
  removed = delayed = 0;
  std::vector<i32> times, common;
  for (i64 k = E - 1; k >= 0; --k) {
    const i64 u = ei[k], v = ej[k];
    // the common neighbourhood of u and v changes only when an edge at u or v
    // appears; between such times a dominating vertex stays dominating (its
    // own neighbourhood only grows)
    times.clear();
    times.push_back((i32)k);
    for (i64 x = 0; x < n; ++x) {
      if (x == u || x == v) continue;
      const i32 a = at[(size_t)(u * n + x)], b = at[(size_t)(v * n + x)];
      if (a != NONE && a > k) times.push_back(a);
      if (b != NONE && b > k) times.push_back(b);
    }
    std::sort(times.begin(), times.end());
    times.erase(std::unique(times.begin(), times.end()), times.end());
    i32 s = NONE;
    for (i32 t : times) {
      common.clear();
      for (i64 x = 0; x < n; ++x)
        if (x != u && x != v && at[(size_t)(u * n + x)] <= t && at[(size_t)(v * n + x)] <= t) common.push_back((i32)x);
      bool dom = false;
      for (i32 w : common) {
        bool all = true;
        for (i32 x : common)
          if (x != w && at[(size_t)(w * n + x)] > t) {
            all = false;
            break;
          }
        if (all) {
          dom = true;
          break;
        }
      }
      if (!dom) {
        s = t;
        break;
      }
    }
    if (s == NONE) {
      slot[k] = -1;
      at[(size_t)(u * n + v)] = at[(size_t)(v * n + u)] = NONE;
      ++removed;
    } else {
      slot[k] = s;
      at[(size_t)(u * n + v)] = at[(size_t)(v * n + u)] = s;
      if (s != k) ++delayed;
    }
  }
  return true;
}

// The same collapse in rounds, the form a GPU kernel can take: the decision
// for edge e = uv reads only the edges that share a triangle with it ((u,x) and
// (v,x) for a common neighbour x) and the edges joining two common neighbours
// (the dominance certificates), later edges at their final times and earlier
// ones at their own. A round decides, all at once, every undecided edge whose
// later such edges are all decided, so each decision sees what the
// last-to-first order above would show it and the slots come out identical
// (common neighbours are taken in the full graph, a superset of every time's).
// rounds = the number of rounds, the length of the longest dependency chain.
bool collapse_edges_rounds(i64 n, const std::vector<i32>& ei, const std::vector<i32>& ej,
                           std::vector<i64>& slot, i64& removed, i64& delayed, i64& rounds) {
  const i64 E = (i64)ei.size();
  const i64 UNDECIDED = -2, DROPPED = -1;
  const i64 NONE = INT64_MAX;
  CSR g = vertex_csr(ei, ej, n);
  auto edge_id = [&](i32 a, i32 b) -> i64 { return edge_rank_lookup(g, a, b); };
  slot.assign(E, UNDECIDED);
  removed = delayed = rounds = 0;
  // per edge: common neighbours x with the ids of (u,x) and (v,x)
  auto commons = [&](i64 e, std::vector<i32>& xs, std::vector<i64>& eu, std::vector<i64>& ev) {
    xs.clear();
    eu.clear();
    ev.clear();
    const i32 u = ei[e], v = ej[e];
    int p = g.ptr[u], q = g.ptr[v];
    while (p < g.ptr[u + 1] && q < g.ptr[v + 1]) {
      if (g.idx[p] < g.idx[q]) ++p;
      else if (g.idx[p] > g.idx[q]) ++q;
      else {
        xs.push_back(g.idx[p]);
        eu.push_back(g.rank[p]);
        ev.push_back(g.rank[q]);
        ++p;
        ++q;
      }
    }
  };
  std::vector<i32> xs;
  std::vector<i64> eu, ev;
  // the edges whose decision e waits for (later edges of its triangles and certificates)
  auto waits_on = [&](i64 e, std::vector<i64>& out) {
    out.clear();
    commons(e, xs, eu, ev);
    for (size_t a = 0; a < xs.size(); ++a) {
      if (eu[a] > e) out.push_back(eu[a]);
      if (ev[a] > e) out.push_back(ev[a]);
      for (size_t b = a + 1; b < xs.size(); ++b) {
        const i64 f = edge_id(xs[a], xs[b]);
        if (f > e) out.push_back(f);
      }
    }
  };
  auto decide = [&](i64 e) -> i64 {
    commons(e, xs, eu, ev);
    auto time_of = [&](i64 f) -> i64 {  // when edge f is present, as e's decision sees it
      if (f < 0) return NONE;
      if (f <= e) return f;
      return slot[f] == DROPPED ? NONE : (slot[f] == UNDECIDED ? f : slot[f]);
    };
    std::vector<i64> tj(xs.size()), times{e};
    for (size_t a = 0; a < xs.size(); ++a) {
      const i64 ta = time_of(eu[a]), tb = time_of(ev[a]);
      tj[a] = (ta == NONE || tb == NONE) ? NONE : std::max(ta, tb);  // x joins the common neighbourhood
      if (tj[a] != NONE && tj[a] > e) times.push_back(tj[a]);
    }
    std::sort(times.begin(), times.end());
    times.erase(std::unique(times.begin(), times.end()), times.end());
    std::vector<size_t> C;
    for (i64 t : times) {
      C.clear();
      for (size_t a = 0; a < xs.size(); ++a)
        if (tj[a] <= t) C.push_back(a);
      bool dom = false;
      for (size_t w : C) {
        bool all = true;
        for (size_t x : C)
          if (x != w && time_of(edge_id(xs[w], xs[x])) > t) {
            all = false;
            break;
          }
        if (all) {
          dom = true;
          break;
        }
      }
      if (!dom) return t;
    }
    return DROPPED;
  };
  std::vector<i64> ready, waits, made;
  i64 left = E;
  while (left > 0) {
    ready.clear();
    for (i64 e = 0; e < E; ++e) {
      if (slot[e] != UNDECIDED) continue;
      waits_on(e, waits);
      bool ok = true;
      for (i64 f : waits)
        if (slot[f] == UNDECIDED) {
          ok = false;
          break;
        }
      if (ok) ready.push_back(e);
    }
    if (ready.empty()) return false;  // cannot happen: the latest undecided edge waits on nothing undecided
    made.resize(ready.size());
    for (size_t a = 0; a < ready.size(); ++a) made[a] = decide(ready[a]);
    for (size_t a = 0; a < ready.size(); ++a) {
      slot[ready[a]] = made[a];
      if (made[a] == DROPPED) ++removed;
      else if (made[a] != ready[a]) ++delayed;
    }
    left -= (i64)ready.size();
    ++rounds;
  }
  return true;
}

// A relaxed round form for a kernel: every round, each edge finds how far it
// can be delayed in the current filtration (the first time, from its current
// one, at which no common neighbour of its ends dominates the others) and the
// edges that certify it (per interval between changes of the common
// neighbourhood: the dominating vertex's edges to u and v and to the other
// common neighbours). Moves whose certificates meet are resolved by
// deterministic reservations: a move reserves its own edge and its certificate
// edges with its priority (later current time first, then higher index) and
// is applied only if it holds every reservation. Applied moves therefore
// never touch one another's certificates, so each stays a delay of a
// dominated edge whatever the others do (the other moves only delay edges,
// which can only shrink the common neighbourhoods), and the rounds repeat
// until no edge can move. The result differs from the last-to-first order but
// is again a sequence of valid moves, so the diagrams are unchanged.
bool collapse_edges_relaxed(i64 n, const std::vector<i32>& ei, const std::vector<i32>& ej,
                            std::vector<i64>& slot, i64& removed, i64& delayed, i64& rounds) {
  const i64 E = (i64)ei.size();
  const i64 NONE = INT64_MAX;
  CSR g = vertex_csr(ei, ej, n);
  std::vector<i64> tm(E);
  std::iota(tm.begin(), tm.end(), (i64)0);
  struct Move {
    i64 e, to, prio;
    std::vector<i64> cert;
  };
  std::vector<Move> moves;
  std::vector<i32> xs;
  std::vector<i64> eu, ev, tj, times, reserve(E, -1);
  std::vector<size_t> C;
  rounds = 0;
  for (;;) {
    moves.clear();
    for (i64 e = 0; e < E; ++e) {
      if (tm[e] == NONE) continue;
      const i32 u = ei[e], v = ej[e];
      xs.clear();
      eu.clear();
      ev.clear();
      for (int p = g.ptr[u], q = g.ptr[v]; p < g.ptr[u + 1] && q < g.ptr[v + 1];) {
        if (g.idx[p] < g.idx[q]) ++p;
        else if (g.idx[p] > g.idx[q]) ++q;
        else {
          xs.push_back(g.idx[p]);
          eu.push_back(g.rank[p]);
          ev.push_back(g.rank[q]);
          ++p;
          ++q;
        }
      }
      tj.assign(xs.size(), NONE);
      times.assign(1, tm[e]);
      for (size_t a = 0; a < xs.size(); ++a) {
        if (tm[eu[a]] == NONE || tm[ev[a]] == NONE) continue;
        tj[a] = std::max(tm[eu[a]], tm[ev[a]]);
        if (tj[a] > tm[e]) times.push_back(tj[a]);
      }
      std::sort(times.begin(), times.end());
      times.erase(std::unique(times.begin(), times.end()), times.end());
      Move m{e, NONE, 0, {}};
      for (i64 t : times) {
        C.clear();
        for (size_t a = 0; a < xs.size(); ++a)
          if (tj[a] <= t) C.push_back(a);
        long dom = -1;
        for (size_t w : C) {
          bool all = true;
          for (size_t x : C) {
            if (x == w) continue;
            const i64 f = edge_rank_lookup(g, xs[w], xs[x]);
            if (f < 0 || tm[f] > t) {
              all = false;
              break;
            }
          }
          if (all) {
            dom = (long)w;
            break;
          }
        }
        if (dom < 0) {
          m.to = t;
          break;
        }
        m.cert.push_back(eu[dom]);
        m.cert.push_back(ev[dom]);
        for (size_t x : C)
          if (x != (size_t)dom) m.cert.push_back(edge_rank_lookup(g, xs[dom], xs[x]));
      }
      if (m.to == tm[e]) continue;  // not dominated at its own time
      m.prio = tm[e] * (E + 1) + e;
      moves.push_back(std::move(m));
    }
    if (moves.empty()) break;
    ++rounds;
    std::fill(reserve.begin(), reserve.end(), (i64)-1);
    for (const Move& m : moves) {
      reserve[m.e] = std::max(reserve[m.e], m.prio);
      for (i64 f : m.cert) reserve[f] = std::max(reserve[f], m.prio);
    }
    for (const Move& m : moves) {
      bool held = reserve[m.e] == m.prio;
      for (i64 f : m.cert) held = held && reserve[f] == m.prio;
      if (held) tm[m.e] = m.to;
    }
  }
  slot.resize(E);
  removed = delayed = 0;
  for (i64 e = 0; e < E; ++e) {
    slot[e] = tm[e] == NONE ? -1 : tm[e];
    if (tm[e] == NONE) ++removed;
    else if (tm[e] != e) ++delayed;
  }
  return true;
}

// [lo, hi) ranges of 0..count over nthreads threads (all cores when 0)
template <typename F>
void parallel_ranges(i64 count, int nthreads, F&& body) {
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nt > count) nt = (int)std::max<i64>(1, count);
  const i64 step = (count + nt - 1) / std::max(nt, 1);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) {
    const i64 lo = t * step, hi = std::min<i64>(count, lo + step);
    if (lo < hi) pool.emplace_back([&body, lo, hi]() { body(lo, hi); });
  }
  body(0, std::min<i64>(count, step));
  for (auto& th : pool) th.join();
}
__attribute__((target("fma"))) inline float fma_hw(float a, float b, float c) { return __builtin_fmaf(a, b, c); }

// H0 and, up to max_dim, H1 and H2 of the sorted filtration in R (edge ranks =
// filtration order, filt = value per rank): persistence.py:160-215.
void run_from_sorted(Result* R, i64 n, const std::vector<float>& filt, int max_dim, int stop_after) {
  const i64 E = (i64)R->edge_i.size();
  boruvka(R->edge_i, R->edge_j, n, R->mst_idx, R->n_components);
  std::vector<float> deaths;
  for (i64 e : R->mst_idx) deaths.push_back(filt[e]);
  std::sort(deaths.begin(), deaths.end());
  for (float x : deaths) {
    R->h0.push_back(0.0f);
    R->h0.push_back(x);
  }
  for (i64 c = 0; c < R->n_components; ++c) {
    R->h0.push_back(0.0f);
    R->h0.push_back(INFINITY);
  }
  if (stop_after == 2 || max_dim == 0) return;
  CSR g = vertex_csr(R->edge_i, R->edge_j, n);
  std::vector<char> mst_mask(E, 0);
  for (i64 e : R->mst_idx) mst_mask[e] = 1;
  Triangles tr = enumerate_triangles(R->edge_i, R->edge_j, g);
  h1_native(*R, n, g, tr, mst_mask, filt);
  if (max_dim >= 2) h2_blocks(*R, g, tr, filt);
}

extern "C" {

// Squared threshold as the reference forms it: double product, then FP32
// (rips.py:125; the kernel argument is an fp32 scalar).
float oracle_threshold_sq(double max_edge_length) {
  return (float)(max_edge_length * max_edge_length);
}

// Full pipeline of persistence.py:77-215 for max_dim 0..2.
// fused: 1 = dist^2 accumulated with fmaf, 0 = separate multiply and add.
// stop_after: 0 = everything, 1 = filtration only, 2 = through H0.
// filt_override: optional per-edge filtration values (sorted edge order, length
// n_override == E) used instead of sqrtf(dist^2); the reference's CPU runs
// take square roots with torch's CPU kernel, which is not always correctly
// rounded, while torch on CUDA and the CUDA path round correctly.
void* oracle_run(const float* pts, int64_t n, int d, double max_edge_length, int max_dim,
                 int fused, int nthreads, int stop_after, const float* filt_override,
                 int64_t n_override) {
  Result* R = new Result();
  const float thr = oracle_threshold_sq(max_edge_length);
  if (n <= 1) {
    if (n == 1) {
      R->h0 = {0.0f, INFINITY};
      R->n_components = 1;
    }
    return R;
  }
  enumerate_edges(pts, n, d, thr, fused, nthreads, R->edge_i, R->edge_j, R->edge_dsq);
  sort_edges(R->edge_i, R->edge_j, R->edge_dsq);
  if (stop_after == 1) return R;
  const i64 E = (i64)R->edge_i.size();
  std::vector<float> filt(E);
  if (filt_override) {
    if (n_override != E) {
      R->error = "filt_override length differs from the edge count";
      return R;
    }
    for (i64 e = 0; e < E; ++e) filt[e] = filt_override[e];
  } else {
    for (i64 e = 0; e < E; ++e) filt[e] = std::sqrt(R->edge_dsq[e]);
  }
  run_from_sorted(R, n, filt, max_dim, stop_after);
  return R;
}

// The same filtration after the edge collapse above (relaxed = 0: last to
// first; 1: the relaxed round form), then H0..H2 of it (the collapse step
// giotto-ph takes before its reduction, persistence.py:48-51). Small inputs
// only (n <= 4096).
void* oracle_run_collapsed(const float* pts, int64_t n, int d, double max_edge_length, int max_dim,
                           int fused, int nthreads, int relaxed) {
  Result* R = new Result();
  const float thr = oracle_threshold_sq(max_edge_length);
  if (n <= 1) {
    if (n == 1) {
      R->h0 = {0.0f, INFINITY};
      R->n_components = 1;
    }
    return R;
  }
  enumerate_edges(pts, n, d, thr, fused, nthreads, R->edge_i, R->edge_j, R->edge_dsq);
  sort_edges(R->edge_i, R->edge_j, R->edge_dsq);
  const i64 E = (i64)R->edge_i.size();
  R->E_full = E;
  std::vector<i64> slot;
  const bool ok = relaxed ? collapse_edges_relaxed(n, R->edge_i, R->edge_j, slot, R->collapse_removed,
                                                   R->collapse_delayed, R->collapse_rounds)
                          : collapse_edges(n, R->edge_i, R->edge_j, slot, R->collapse_removed, R->collapse_delayed);
  if (!ok) {
    R->error = "oracle_run_collapsed: n > 4096";
    return R;
  }
  std::vector<float> filt0(E);
  for (i64 e = 0; e < E; ++e) filt0[e] = std::sqrt(R->edge_dsq[e]);
  std::vector<i64> keep;
  for (i64 e = 0; e < E; ++e)
    if (slot[e] >= 0) keep.push_back(e);
  std::stable_sort(keep.begin(), keep.end(), [&](i64 a, i64 b) { return slot[a] < slot[b]; });
  std::vector<i32> ni, nj;
  std::vector<float> nd, filt;
  for (i64 e : keep) {
    ni.push_back(R->edge_i[e]);
    nj.push_back(R->edge_j[e]);
    nd.push_back(R->edge_dsq[e]);
    filt.push_back(filt0[slot[e]]);
  }
  R->edge_i.swap(ni);
  R->edge_j.swap(nj);
  R->edge_dsq.swap(nd);
  run_from_sorted(R, n, filt, max_dim, 0);
  return R;
}

// Slots of the edge collapse computed both ways (last to first, and in
// rounds) on the sorted filtration of the points; arrays "slot_seq" and
// "slot_rounds", scalar "collapse_rounds". Small inputs only (n <= 4096).
void* oracle_collapse_slots(const float* pts, int64_t n, int d, double max_edge_length, int fused,
                            int nthreads) {
  Result* R = new Result();
  if (n <= 1) return R;
  enumerate_edges(pts, n, d, oracle_threshold_sq(max_edge_length), fused, nthreads, R->edge_i, R->edge_j,
                  R->edge_dsq);
  sort_edges(R->edge_i, R->edge_j, R->edge_dsq);
  R->E_full = (i64)R->edge_i.size();
  i64 rm = 0, dl = 0;
  if (!collapse_edges(n, R->edge_i, R->edge_j, R->slot_seq, rm, dl) ||
      !collapse_edges_rounds(n, R->edge_i, R->edge_j, R->slot_rounds, R->collapse_removed, R->collapse_delayed,
                             R->collapse_rounds)) {
    R->error = "oracle_collapse_slots: n > 4096 or no edge ready";
  }
  return R;
}

// dist^2 of given pairs (i, j) with the chain of enumerate_edges (fused or
// not): the arithmetic of edge_kernel.py:111-123 for each pair, so that a
// candidate edge list can be checked bit for bit without enumerating all
// n(n-1)/2 pairs.
void oracle_edge_dsq(const float* pts, int64_t n, int d, const int32_t* ei, const int32_t* ej, int64_t E,
                     int fused, int nthreads, float* out) {
  (void)n;
  const bool hw_fma = __builtin_cpu_supports("fma");
  auto body = [&](i64 lo, i64 hi) {
    for (i64 e = lo; e < hi; ++e) {
      const float* x = pts + (i64)ei[e] * d;
      const float* y = pts + (i64)ej[e] * d;
      float acc = 0.0f;
      for (int k = 0; k < d; ++k) {
        const float df = x[k] - y[k];
        acc = fused ? (hw_fma ? fma_hw(df, df, acc) : __builtin_fmaf(df, df, acc)) : acc + df * df;
      }
      out[e] = acc;
    }
  };
  parallel_ranges(E, nthreads, body);
}

// Every pair (r, j), j != r, of the rows r listed in `rows` with dist^2 below
// the threshold (chain of enumerate_edges), written as edges (min, max) with
// their dist^2, rows in the given order, j ascending: the rows' slice of the
// edge set of edge_kernel.py:152 for a completeness check of a GPU edge list.
void* oracle_row_edges(const float* pts, int64_t n, int d, double max_edge_length, const int32_t* rows,
                       int64_t m, int fused, int nthreads) {
  Result* R = new Result();
  const float thr = oracle_threshold_sq(max_edge_length);
  const bool hw_fma = __builtin_cpu_supports("fma");
  std::vector<std::vector<i32>> vi(m), vj(m);
  std::vector<std::vector<float>> vd(m);
  auto body = [&](i64 lo, i64 hi) {
    for (i64 q = lo; q < hi; ++q) {
      const i64 r = rows[q];
      const float* x = pts + r * d;
      for (i64 j = 0; j < n; ++j) {
        if (j == r) continue;
        // the kernel's operand order: the lower index is the source row
        const float* a = j < r ? pts + j * d : x;
        const float* b = j < r ? x : pts + j * d;
        float acc = 0.0f;
        for (int k = 0; k < d; ++k) {
          const float df = a[k] - b[k];
          acc = fused ? (hw_fma ? fma_hw(df, df, acc) : __builtin_fmaf(df, df, acc)) : acc + df * df;
        }
        if (acc < thr) {
          vi[q].push_back((i32)std::min<i64>(r, j));
          vj[q].push_back((i32)std::max<i64>(r, j));
          vd[q].push_back(acc);
        }
      }
    }
  };
  parallel_ranges(m, nthreads, body);
  for (i64 q = 0; q < m; ++q) {
    R->edge_i.insert(R->edge_i.end(), vi[q].begin(), vi[q].end());
    R->edge_j.insert(R->edge_j.end(), vj[q].begin(), vj[q].end());
    R->edge_dsq.insert(R->edge_dsq.end(), vd[q].begin(), vd[q].end());
  }
  return R;
}

// The pipeline from a given edge list (any order): the edges are first put
// in the reference kernel's emission order (32-point tiles (I, J), I <= J,
// row-major over the flattened nb x nb grid, row-major inside a tile:
// edge_kernel.py:134-149,208-210), then sorted by the packed key stably
// (rips.py:30-50,188-202), then H0..H2 as oracle_run does. With the edge
// set of edge_kernel.py this is oracle_run without the O(n^2 d) enumeration,
// for checking large clouds whose edge list was checked separately.
void* oracle_run_edges(const int32_t* ei, const int32_t* ej, const float* edsq, int64_t E, int64_t n,
                       int max_dim) {
  Result* R = new Result();
  if (n <= 1) {
    if (n == 1) {
      R->h0 = {0.0f, INFINITY};
      R->n_components = 1;
    }
    return R;
  }
  const i64 B = 32, nb = (n + B - 1) / B;
  std::vector<u64> ek(E);
  for (i64 e = 0; e < E; ++e) {
    const i64 i = ei[e], j = ej[e];
    if (!(0 <= i && i < j && j < n)) {
      R->error = "oracle_run_edges: an edge is not (i, j) with 0 <= i < j < n";
      return R;
    }
    ek[e] = ((u64)((i / B) * nb + j / B) << 10) | (u64)((i % B) * B + j % B);
  }
  std::vector<i64> perm(E);
  std::iota(perm.begin(), perm.end(), 0);
  std::sort(perm.begin(), perm.end(), [&](i64 a, i64 b) { return ek[a] < ek[b]; });
  R->edge_i.resize(E);
  R->edge_j.resize(E);
  R->edge_dsq.resize(E);
  for (i64 k = 0; k < E; ++k) {
    R->edge_i[k] = ei[perm[k]];
    R->edge_j[k] = ej[perm[k]];
    R->edge_dsq[k] = edsq[perm[k]];
  }
  sort_edges(R->edge_i, R->edge_j, R->edge_dsq);
  std::vector<float> filt(E);
  for (i64 e = 0; e < E; ++e) filt[e] = std::sqrt(R->edge_dsq[e]);
  run_from_sorted(R, n, filt, max_dim, 0);
  return R;
}

void oracle_free(void* h) { delete static_cast<Result*>(h); }

// Returns a pointer to the named array and its element count (0 if empty).
// dtype codes: 1 = int32, 2 = int64, 3 = float32.
const void* oracle_get(void* h, const char* name, int64_t* count, int* dtype) {
  Result* R = static_cast<Result*>(h);
  std::string s(name);
#define ARR(nm, vec, code)              \
  if (s == nm) {                        \
    *count = (int64_t)R->vec.size();    \
    *dtype = code;                      \
    return R->vec.data();               \
  }
  ARR("edge_i", edge_i, 1)
  ARR("edge_j", edge_j, 1)
  ARR("edge_dsq", edge_dsq, 3)
  ARR("mst_idx", mst_idx, 2)
  ARR("h0", h0, 3)
  ARR("tri_max_rank_sorted", tri_max_rank_sorted, 1)
  ARR("ap_births", ap_births, 1)
  ARR("ap_deaths", ap_deaths, 1)
  ARR("res_births", res_births, 1)
  ARR("res_deaths", res_deaths, 1)
  ARR("ess_births", ess_births, 1)
  ARR("h1_all_pivots", h1_all_pivots, 1)
  ARR("h1", h1, 3)
  ARR("h2", h2, 3)
  ARR("h2_births", h2_births, 1)
  ARR("h2_deaths", h2_deaths, 1)
  ARR("h2_ess", h2_ess, 1)
  ARR("slot_seq", slot_seq, 2)
  ARR("slot_rounds", slot_rounds, 2)
#undef ARR
  *count = -1;
  *dtype = 0;
  return nullptr;
}

const char* oracle_error(void* h) { return static_cast<Result*>(h)->error.c_str(); }

int64_t oracle_scalar(void* h, const char* name) {
  Result* R = static_cast<Result*>(h);
  std::string s(name);
  if (s == "E") return (int64_t)R->edge_i.size();
  if (s == "n_components") return R->n_components;
  if (s == "T") return R->T;
  if (s == "Q") return R->Q;
  if (s == "cofacet_nnz") return R->cofacet_nnz;
  if (s == "n_apparent") return R->n_apparent;
  if (s == "residual") return R->residual;
  if (s == "xor_ops") return R->xor_ops;
  if (s == "xor_max") return R->xor_max;
  if (s == "xor_elems") return R->xor_elems;
  if (s == "crit_path") return R->crit_path;
  if (s == "col_max") return R->col_max;
  if (s == "E_full") return R->E_full;
  if (s == "collapse_removed") return R->collapse_removed;
  if (s == "collapse_delayed") return R->collapse_delayed;
  if (s == "collapse_rounds") return R->collapse_rounds;
  return -1;
}

}  // extern "C"
