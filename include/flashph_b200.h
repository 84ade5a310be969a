/*
 * flashph_b200.h -- C ABI of the B200 (sm_100a) CUDA library for exact
 * Vietoris-Rips persistent homology (H0/H1/H2 over Z/2).
 *
 * Every entry point takes raw device pointers, element counts and a CUDA
 * stream (cudaStream_t passed as void*), enqueues its kernels on that stream
 * and returns a status code without synchronising. Outputs are written into
 * caller-allocated device buffers; functions that need scratch memory take a
 * (workspace, workspace_bytes) pair whose size is given by the matching
 * *_workspace_bytes() query. Counts that the caller needs on the host
 * (edges, triangles, tetrahedra, diagram rows) are written to device
 * memory; the caller copies them back when it needs them.
 *
 * The functions mirror the internal seams of the reference implementation
 * (ot-triton-lab/flash-ph, Python); each declaration names the reference
 * function it replaces. Nothing here calls back into Python, Triton or Numba.
 */
#ifndef FLASHPH_B200_H_
#define FLASHPH_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PH_OK 0
#define PH_ERR_CUDA 1        /* a CUDA launch or runtime call failed          */
#define PH_ERR_ARG 2         /* invalid argument or workspace too small      */
#define PH_ERR_CAPACITY 3    /* an output buffer was too small (count is set) */
#define PH_ERR_ITER_LIMIT 4  /* a bounded device loop hit its iteration cap  */
#define PH_ERR_POOL 5        /* reduction column pool exhausted              */
#define PH_ERR_OVERFLOW 6    /* a count does not fit the index type          */
#define PH_ERR_LIMIT 7       /* a user limit was exceeded (ValueError text)  */

/* Library version (major*10000 + minor*100 + patch). No counterpart in the
 * reference (library utility), like the two functions below. */
int ph_version(void);

/* Last CUDA error string seen by the library on this thread ("" if none). */
const char* ph_last_error(void);

/* Number of kernels this library has launched in this process so far. */
unsigned long long ph_launch_count(void);

/* Kernels launched from the calling host thread are chained with
 * programmatic dependent launch (the next kernel's blocks are scheduled while
 * the current one drains; each kernel waits on the device for its
 * predecessor). On by default; enable = 0 switches it off for this thread,
 * e.g. for threads that drive several streams at once, where blocks scheduled
 * early hold SMs that another stream's kernels could use. No counterpart in
 * the reference (a launch policy of this library). */
void ph_set_dependent_launch(int32_t enable);

/* Test-only limits of the Z/2 reduction, process-wide: the most steps
 * (column additions and pivot claims) one column may take before
 * ph_reduce reports PH_ERR_ITER_LIMIT (default 2^24), and a cap on the
 * reduction pool of the native calls' first attempt (a pool that runs out is
 * retried 4x larger). 0 restores a default. No counterpart in the reference
 * (whose Numba loops have no such bounds); used to exercise the failure paths
 * without a device fault. */
void ph_set_reduce_limits(int64_t max_steps, int64_t first_pool_entries);

/* Measurement probe: one thread follows `hops` links of the cycle `next`
 * (next[i] is the index of the next entry; a random cycle over a buffer that
 * fits L2) from `start`, once to warm L2 and once timed; d_out[0] receives
 * the timed lap's nanoseconds (device memory, 2 entries). The latency of one
 * dependent L2 load, the unit of the reduction's latency bound. No
 * counterpart in the reference. */
int ph_probe_l2_chase(const uint32_t* next, int32_t hops, uint32_t start, unsigned long long* d_out,
                      void* stream);

/* ---- filtration -------------------------------------------------------- */

/* One point cloud of a batch. A batch is the disjoint union of its clouds:
 * cloud c's vertices get the global indices vbase .. vbase + n - 1, and all
 * later stages (adjacency, forest, triangles, tetrahedra, reduction) work on
 * global indices unchanged, since no simplex spans two clouds. */
typedef struct ph_cloud_seg {
  int64_t pt_off;   /* offset, in floats, of the cloud's first coordinate      */
  int64_t vbase;    /* global index of the cloud's first vertex                */
  int64_t tile_off; /* first edge-enumeration work item (ph_cloud_tiles each)  */
  int32_t n;        /* points in the cloud                                      */
  int32_t d;        /* dimension                                                */
  float thr_sq;     /* fp32(max_edge_length^2)                                  */
  int32_t max_dim;  /* 0, 1 or 2                                                */
} ph_cloud_seg;

/* All pairs i < j with sum_k (x_ik - x_jk)^2 < thr_sq, the squares
 * accumulated over k = 0..d-1 in order, one fused multiply-add per step,
 * in FP32. Replaces kernels/edge_kernel.py:152 direct_edge_enumerate (its
 * count and emit kernels, edge_kernel.py:23-149). Edges are written in an
 * unspecified order to out_i/out_j/out_dsq up to `capacity`; *d_count (u64,
 * device) receives the total, which may exceed capacity (then rerun with a
 * larger buffer). pts: (n, d) float32 row-major. */
int ph_edges_enumerate(const float* pts, int64_t n, int32_t d, float thr_sq, int32_t* out_i,
                       int32_t* out_j, float* out_dsq, int64_t capacity,
                       unsigned long long* d_count, void* stream);

/* Edge-enumeration work items (128 x 128 point tiles, i-tile <= j-tile) of a
 * cloud of n points: the counterpart of the reference kernel's program grid
 * (kernels/edge_kernel.py:208-210, 32-point tiles). */
int64_t ph_cloud_tiles(int64_t n);

/* ph_edges_enumerate over a batch: segs (device) holds nsegs clouds ordered
 * by tile_off; ntiles is the total number of work items. Vertex indices
 * are written as global indices. Replaces one kernels/edge_kernel.py:152
 * direct_edge_enumerate call per cloud (rips.py:151-159); the reference has
 * no batched form. */
int ph_batch_edges_enumerate(const float* pts, const ph_cloud_seg* segs, int32_t nsegs, int64_t ntiles,
                             int32_t* out_i, int32_t* out_j, float* out_dsq, int64_t capacity,
                             unsigned long long* d_count, void* stream);

/* ph_batch_edges_enumerate with a tensor-core screen (d <= 252), also
 * replacing kernels/edge_kernel.py:152 direct_edge_enumerate: every
 * cloud is centred on its mean and rounded to BF16, 128 x 128 point tiles
 * of an augmented Gram matrix (|y_i|^2 + |y_j|^2 - 2 y_i.y_j) are formed by
 * tcgen05.mma into tensor memory, and each value is compared with the
 * threshold widened by a certified bound on the BF16 rounding of the points
 * and the FP32 accumulation; the surviving pairs are recomputed with the
 * exact FP32 chain of ph_edges_enumerate. The edge set and dist^2 bits are
 * those of the direct kernel (the emission order differs, as it does between
 * runs of either kernel). blk_off (nsegs+1, device): per-cloud offsets of
 * 128-point blocks, nblocks their total; N the number of points; max_d the
 * largest d. d_status gets PH_ERR_ITER_LIMIT if a bounded wait for the
 * tensor cores gives up. d_stats (2 x u64, device, may be null) accumulates
 * the pairs that passed the screen and the pairs of tiles recomputed without
 * it (non-finite or huge coordinates, huge thresholds).
 * Replaces the same call site as ph_batch_edges_enumerate. */
size_t ph_edges_screened_workspace_bytes(int64_t N, int32_t nsegs, int32_t max_d);
int ph_batch_edges_enumerate_screened(const float* pts, const ph_cloud_seg* segs, int32_t nsegs,
                                      int64_t ntiles, int32_t max_d, int64_t N, const int64_t* blk_off,
                                      int64_t nblocks, int32_t* out_i, int32_t* out_j, float* out_dsq,
                                      int64_t capacity, unsigned long long* d_count, int* d_status,
                                      unsigned long long* d_stats, void* workspace, size_t workspace_bytes,
                                      void* stream);

/* Orders E edges by the reference's packed key
 *   (float bits of dist^2) << 32 | (j(j-1)/2 + i) & 0xFFFFFFFF
 * stably with respect to the reference kernel's emission order (tiles of 32
 * points in row-major order, row-major inside a tile), which only matters
 * when the 32-bit colex part collides (n > 92682). Replaces rips.py:30-50
 * _pack_sort_key and the stable argsort of rips.py:189-195. Inputs are the
 * unsorted edges of ph_edges_enumerate; outputs are separate buffers. */
size_t ph_edges_sort_workspace_bytes(int64_t E);
int ph_edges_sort(const int32_t* in_i, const int32_t* in_j, const float* in_dsq, int64_t E,
                  int64_t n, int32_t* out_i, int32_t* out_j, float* out_dsq, void* workspace,
                  size_t workspace_bytes, void* stream);

/* ph_edges_sort for callers that cannot allocate device memory (their HBM
 * is owned by another allocator or a fixed budget). No counterpart in the
 * reference. Takes only inputs and outputs; its scratch is a 13 MiB static
 * device array held by every GPU that loads the library, so E may not exceed
 * ph_edges_sort_noalloc_max_edges() (2^19); larger E returns PH_ERR_CAPACITY
 * with a message in ph_last_error(). The array's device address is looked up
 * on the first call on each device. All calls share the array: calls whose
 * work overlaps on the GPU race and must be ordered by the caller. */
int64_t ph_edges_sort_noalloc_max_edges(void);
int ph_edges_sort_noalloc(const int32_t* in_i, const int32_t* in_j, const float* in_dsq, int64_t E,
                          int64_t n, int32_t* out_i, int32_t* out_j, float* out_dsq, void* stream);

/* Per-vertex adjacency with two half-edges per edge, rows sorted by
 * neighbour index, each entry carrying the edge rank (its position in the
 * sorted edge list). Replaces rips.py:53-95 _build_vertex_csr.
 * adj_ptr: n+1, adj_idx/adj_rank: 2E. */
size_t ph_vertex_csr_workspace_bytes(int64_t E);
int ph_vertex_csr(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                  int32_t* adj_ptr, int32_t* adj_idx, int32_t* adj_rank, void* workspace,
                  size_t workspace_bytes, void* stream);

/* Square root of each dist^2 (correctly rounded), the edge filtration
 * values of reduce_h1_gpu.py:479. */
int ph_sqrt_f32(const float* in, float* out, int64_t count, void* stream);

/* ---- H0 ------------------------------------------------------------------ */

/* Minimum spanning forest under the integer weights edge_rank = position
 * (ties impossible), as boruvka.py:17 gpu_boruvka_mst computes it. mst_mask[e]
 * is set to 1 for forest edges; comp[v] receives the smallest vertex index of
 * v's component (the reference's root labels); *d_ncomp (int64, device) the
 * number of components. d_status (int, device) gets PH_ERR_ITER_LIMIT if
 * the bounded round loop does not converge. */
size_t ph_boruvka_workspace_bytes(int64_t n, int64_t E);
int ph_boruvka_mst(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                   uint8_t* mst_mask, int32_t* comp, int64_t* d_ncomp, int* d_status,
                   void* workspace, size_t workspace_bytes, void* stream);

/* H0 rows of persistence.py:169-192: (0, sqrt(dist^2)) for the forest edges
 * in ascending order, then ncomp rows (0, inf); n rows in total.
 * out_rows: n x 2 float32. */
size_t ph_h0_rows_workspace_bytes(int64_t E);
int ph_h0_rows(const float* edge_filt, const uint8_t* mst_mask, int64_t E, int64_t n,
               float* out_rows, void* workspace, size_t workspace_bytes, void* stream);

/* ---- triangles (H1 cofacets) -------------------------------------------- */

/* For every edge m = (a, b) (by rank): tri_cnt[m] = number of w with edges
 * (a,w), (b,w) both ranked below m (the triangles whose largest edge is m),
 * cof_cnt[m] = number of common neighbours of a and b (the triangles
 * containing m). Offsets are exclusive scans (E+1 entries, last = total).
 * Together with ph_triangles_emit this replaces triangle_kernel.py:288
 * triangle_enumerate and the face-rank lookup and triangle ordering of
 * reduce_h1_gpu.py:65-100,509-521: triangles come out already ordered by
 * (largest edge rank, colex), which for a fixed largest edge equals the order
 * of the third vertex, so the global rank of a triangle is E + its position. */
size_t ph_triangles_count_workspace_bytes(int64_t E);
int ph_triangles_count(const int32_t* edge_i, const int32_t* edge_j, int64_t E,
                       const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                       int64_t* tri_off, int64_t* cof_off, void* workspace,
                       size_t workspace_bytes, void* stream);

/* Exact number of triangles of the graph (the sum of ph_triangles_count's
 * per-edge counts), without ranks: each triangle x < y < z is found once from
 * a shared-memory bitmap of N(x). Work ~ sum over vertices of deg^2 / 6
 * bitmap tests, far below the per-edge count's searches on dense graphs; used
 * to check the reference's max_triangles limit (triangle_kernel.py:377-381)
 * before the per-edge pass. n <= ph_triangles_total_max_vertices(); d_next:
 * one int of device scratch. */
int64_t ph_triangles_total_max_vertices(void);
int ph_triangles_total(const int32_t* adj_ptr, const int32_t* adj_idx, int64_t n,
                       unsigned long long* d_total, int* d_next, void* stream);

/* ph_triangles_total from the unsorted edges (i < j, any order), without the
 * adjacency: an upper adjacency (row i lists the j of every edge (i, j)) is
 * built by counting, then the same bitmap pass runs. The total the count pass
 * of triangle_kernel.py:288 triangle_enumerate checks against max_triangles
 * (triangle_kernel.py:377-381), for a call that may be over the limit, before
 * any filtration order exists. n <= ph_triangles_total_max_vertices(). */
size_t ph_triangles_total_edges_workspace_bytes(int64_t E, int64_t n);
int ph_triangles_total_edges(const int32_t* edge_i, const int32_t* edge_j, int64_t E, int64_t n,
                             unsigned long long* d_total, void* workspace, size_t workspace_bytes, void* stream);

/* ph_triangles_total per cloud of a batch's union graph (sorted rows of
 * ph_vertex_csr over global vertices): vertex a's triangles go to
 * d_per[vcloud[a]] (nclouds entries, zeroed here), and only the vertices of
 * clouds with want[cloud] != 0 are visited. The batch form of the limit check
 * of triangle_kernel.py:377-381: clouds that may be over max_triangles are
 * counted exactly before the per-edge pass, which then skips those over it.
 * n <= ph_triangles_total_max_vertices(); d_next: one int of device scratch. */
int ph_batch_triangles_total(const int32_t* adj_ptr, const int32_t* adj_idx, int64_t n, const int32_t* vcloud,
                             const uint8_t* want, int32_t nclouds, unsigned long long* d_per, int* d_next,
                             void* stream);

/* Writes, for every triangle in global order, its largest edge tri_m, third
 * vertex tri_w and the ranks of its two other edges (a,w) and (b,w): the emit
 * pass of triangle_kernel.py:288 triangle_enumerate with the face ranks of
 * reduce_h1_gpu.py:65-100. */
int ph_triangles_emit(const int32_t* edge_i, const int32_t* edge_j, int64_t E,
                      const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                      const int64_t* tri_off, int32_t* tri_m, int32_t* tri_w, int32_t* tri_fa,
                      int32_t* tri_fb, void* stream);

/* ---- tetrahedra (H2 cofacets) ------------------------------------------- */

/* For every edge m: the tetrahedra whose largest edge is m, i.e. pairs
 * p < q of third vertices of triangles with largest edge m such that (p,q)
 * is an edge ranked below m. Ordered by (largest edge rank, p, q).
 * Replaces triangle_kernel.py:402 tetrahedra_enumerate (count and emit
 * kernels, triangle_kernel.py:152-270). tet_off: E+1. edge_enable
 * (optional, E bytes): only edges with a non-zero flag get tetrahedra (in a
 * batch, the edges of clouds that asked for H2). */
size_t ph_tets_count_workspace_bytes(int64_t E);
int ph_tets_count(const int64_t* tri_off, const int32_t* tri_w, int64_t E,
                  const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                  const uint8_t* edge_enable, int64_t* tet_off, void* workspace,
                  size_t workspace_bytes, void* stream);

/* Writes per tetrahedron its largest edge and the local indices (triangle
 * global rank - E) of its four triangle faces (the emit kernel of
 * triangle_kernel.py:402 tetrahedra_enumerate with the face lookup of
 * apparent_pair_h2_kernel.py:37-49). tet_faces: Q x 4.
 * d_status gets PH_ERR_ARG if a face triangle cannot be found (inconsistent
 * inputs). */
int ph_tets_emit(const int32_t* edge_i, const int32_t* edge_j, int64_t E, const int64_t* tri_off,
                 const int32_t* tri_w, const int32_t* tri_fa, const int32_t* tri_fb,
                 const int32_t* adj_ptr, const int32_t* adj_idx, const int32_t* adj_rank,
                 const uint8_t* edge_enable, const int64_t* tet_off, int32_t* tet_m,
                 int32_t* tet_faces, int* d_status, void* stream);

/* ---- coboundary columns and reduction ----------------------------------- */

/* Cofacet CSR: for each of n_faces faces, the global ranks
 * (row_base + simplex index) of the simplices containing it, ascending.
 * faces: S x k local face indices of each simplex, simplices given in
 * ascending order. For triangles (k = 3) the faces are (tri_m, tri_fa,
 * tri_fb) passed as three separate arrays through faces_soa; for tetrahedra
 * (k = 4) tet_faces is passed as faces_aos. Replaces reduce_h1_gpu.py:107
 * _build_cofacet_csr_h1. cof_off: n_faces + 1, cof_data: k*S. */
size_t ph_cofacet_csr_workspace_bytes(int64_t S, int32_t k);
int ph_cofacet_csr(const int32_t* faces_aos, const int32_t* f0, const int32_t* f1,
                   const int32_t* f2, int32_t k, int64_t S, int64_t n_faces, int32_t row_base,
                   int32_t* cof_off, int32_t* cof_data, void* workspace, size_t workspace_bytes,
                   void* stream);

/* The H1 cofacet CSR of ph_cofacet_csr (k = 3, faces f0/f1/f2 per triangle)
 * without its sort: row_off (n_faces + 1, int64) are the rows' offsets known
 * beforehand -- the cofacet offsets ph_triangles_count writes (one entry per
 * common neighbour of an edge's ends), masked like the triangles when some
 * are cleared -- so every triangle's rank is scattered straight into its
 * three rows and each row is then sorted in shared memory (a warp a row up to
 * 1024 entries, a block a row up to ph_cofacet_rows3_max_row()). max_row:
 * the longest row (ph_max_count on row_off); longer rows return PH_ERR_ARG
 * (use ph_cofacet_csr). Same output as ph_cofacet_csr; replaces the same
 * reduce_h1_gpu.py:107 _build_cofacet_csr_h1. d_status gets PH_ERR_ARG if a
 * row turns out longer than max_row. */
int32_t ph_cofacet_rows3_max_row(void);
size_t ph_cofacet_rows3_workspace_bytes(int64_t n_faces);
int ph_cofacet_rows3(const int32_t* f0, const int32_t* f1, const int32_t* f2, int64_t S, int64_t n_faces,
                     int32_t row_base, const int64_t* row_off, int32_t max_row, int32_t* cof_off, int32_t* cof_data,
                     int* d_status, void* workspace, size_t workspace_bytes, void* stream);
/* *d_out = max over i < n of off[i + 1] - off[i] (int64, device): the longest
 * row of an exclusive-scan offset array. Bookkeeping with no counterpart. */
int ph_max_count(const int64_t* off, int64_t n, int64_t* d_out, void* stream);

/* For every simplex: the largest global rank (face_base + face index) among
 * its faces that are not skipped, -1 if all are skipped. This is the
 * cofacet_max_face of reduce_h1_gpu.py:186-197 / cohomology_general.py:50-61. */
int ph_cof_max_face(const int32_t* faces_aos, const int32_t* f0, const int32_t* f1,
                    const int32_t* f2, int32_t k, int64_t S, int32_t face_base,
                    const uint8_t* skip, int32_t* cmf, void* stream);

/* Z/2 cohomology reduction of K columns (faces) over their cofacet rows,
 * processed in the reference's order (descending rank), pivot = smallest
 * cofacet rank. Apparent pairs (the column is the largest non-skipped face of
 * its youngest cofacet) are detected first (reduce_h1_gpu.py:159-223); the
 * remaining columns are reduced on the GPU lock-free, one warp per column:
 * a column adds the column owning its pivot while that owner was processed
 * earlier (larger index), then claims the pivot with an atomic maximum,
 * taking over any later-processed column it displaces. The pivots, and so
 * the pairs and the essential columns, are those of the serial reduction
 * (cohomology_general.py:202-371).
 * col_state[c]: 0 skipped, 1 apparent, 2 reduced to a pivot, 3 essential.
 * col_piv[c]: pivot global rank (states 1 and 2) or -1.
 * pool: scratch for reduced columns, pool_cap int32 entries.
 * span: the most rows one column's entries can span (its rows all lie in a
 * range of span consecutive ranks: in a batch, the largest row count of one
 * cloud); 0 or R for a single cloud. Working columns that become bitmaps
 * need only that many bits.
 * d_info (int64 x 4, device): [residual columns, column additions, pool
 * entries used, takeovers].
 * d_status: PH_ERR_POOL or PH_ERR_ITER_LIMIT on failure. */
size_t ph_reduce_workspace_bytes(int64_t K, int64_t R, int64_t span);
int ph_reduce(const int32_t* cof_off, const int32_t* cof_data, int64_t K, int32_t col_base,
              int64_t R, int32_t row_base, int64_t span, const uint8_t* skip, const int32_t* row_cmf,
              int32_t* col_state, int32_t* col_piv, int32_t* pool, int64_t pool_cap,
              int64_t* d_info, int* d_status, void* workspace, size_t workspace_bytes,
              void* stream);

/* Marks the rows that are pivots of reduced or apparent columns (the H1
 * pivots that clear H2 columns, cohomology_general.py:171-173,635). */
int ph_mark_pivots(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                   uint8_t* row_flag, int64_t R, void* stream);

/* Persistence rows in the reference's order (reduce_h1_gpu.py:574-604):
 * apparent pairs by ascending column, then reduced pairs and essential
 * columns by descending column, pairs kept when death > birth (as float32),
 * then a stable sort by birth. Columns in index order have non-decreasing
 * birth values, so the sort only reorders runs of equal birth, which are
 * ordered in place; no sort is run. Column c's value is filt[col_m ? col_m[c] : c],
 * row r's value is filt[row_m[r]]. out_rows: capacity K x 2; *d_nrows (int64). */
size_t ph_persistence_rows_workspace_bytes(int64_t K);
int ph_persistence_rows(const int32_t* col_state, const int32_t* col_piv, int64_t K,
                        int32_t row_base, const float* filt, const int32_t* col_m,
                        const int32_t* row_m, float* out_rows, int64_t* d_nrows, void* workspace,
                        size_t workspace_bytes, void* stream);

/* ---- the whole call --------------------------------------------------------- */

/* rips_persistence for one cloud, every stage on `stream`: points (device,
 * n x d float32, n >= 2), max_edge_length (edges keep dist^2 <
 * fp32(max_edge_length^2)), max_dim 0..2, the reference's max_triangles /
 * max_tetrahedra limits, edge_mode 0 (tensor-core screen when 8 <= d <= 252),
 * 1 (screen), 2 (direct kernel). On success *out holds the diagrams on the
 * device; read them with ph_result_rows / ph_result_copy and release with
 * ph_result_free. A limit exceeded returns PH_ERR_LIMIT with the reference's
 * ValueError message in ph_last_error(). The host waits at most four times
 * (edge, triangle and tetrahedron counts, reduction statuses).
 * Replaces persistence.py:77-215 rips_persistence (the n >= 2 path). */
typedef struct ph_result ph_result;
int ph_rips_persistence(const float* points, int64_t n, int32_t d, double max_edge_length, int32_t max_dim,
                        int64_t max_triangles, int64_t max_tetrahedra, int32_t edge_mode, ph_result** out,
                        void* stream);
/* Accessors of ph_rips_persistence's result, the list of (K, 2) diagrams
 * that persistence.py:77 returns.
 * rows of diagram dim (0..max_dim), -1 if out of range */
int64_t ph_result_rows(const ph_result* result, int32_t dim);
/* run statistics: 0 edges, 1 triangles, 2 tetrahedra, 3 H1 column additions,
 * 4 H2 column additions */
int64_t ph_result_stat(const ph_result* result, int32_t k);
/* copies diagram dim (rows x 2 float32) to dst, device or host memory, on
 * `stream` (any stream: when it is not the run's stream, the run's stream is
 * made to wait for the copy, so that ph_result_free cannot release the rows
 * before the copy has read them) */
int ph_result_copy(const ph_result* result, int32_t dim, float* dst, int32_t to_host, void* stream);
/* copies every diagram, dim 0 first, into one buffer of sum(rows) x 2 float32
 * (stream rule of ph_result_copy) */
int ph_result_copy_all(const ph_result* result, float* dst, int32_t to_host, void* stream);
/* releases the diagrams and the run's intermediate buffers (stream-ordered, on
 * the stream of the run, after every copy queued before it) */
void ph_result_free(ph_result* result);

/* ---- the whole call for a batch of clouds ------------------------------------ */

/* rips_persistence for every cloud of a batch in one call (the reference has
 * no batched API; this replaces one persistence.py:77-215 call per cloud):
 * points[c] (device, n[c] x d[c] float32, n[c] >= 2), max_edge_length[c],
 * max_dim[c] (0..2; H2 needs n[c] < 65536), the reference's per-call limits,
 * edge_mode as in ph_rips_persistence (0: the tensor-core screen when the
 * largest d is in [8, 252]). The clouds run as one disjoint union on
 * `stream`; the host waits four times whatever their number. A cloud over a
 * limit gets status PH_ERR_LIMIT and the reference's ValueError text
 * (ph_batch_result_status / _message); the others are unaffected, and every
 * cloud's diagrams equal ph_rips_persistence on it alone, bit for bit.
 * Returns PH_ERR_CAPACITY, with *out set and the per-cloud counts filled,
 * when the union's simplices exceed the int32 rank range or, for more than
 * one cloud, max_batch_simplices (triangles, then triangles + tetrahedra;
 * 0: no budget): the caller splits the batch (ph_batch_result_stat gives each
 * cloud's edges and triangles) and frees *out. */
typedef struct ph_batch_result ph_batch_result;
int ph_rips_persistence_batch(const float* const* points, const int64_t* n, const int32_t* d,
                              const double* max_edge_length, const int32_t* max_dim, int32_t nclouds,
                              int64_t max_triangles, int64_t max_tetrahedra, int32_t edge_mode,
                              int64_t max_batch_simplices, ph_batch_result** out, void* stream);
/* PH_OK or PH_ERR_LIMIT for cloud c, and the limit's message ("" if none) */
int32_t ph_batch_result_status(const ph_batch_result* result, int32_t cloud);
const char* ph_batch_result_message(const ph_batch_result* result, int32_t cloud);
/* per-cloud counts: k = 0 edges, 1 triangles, 2 tetrahedra (-1: not counted) */
int64_t ph_batch_result_stat(const ph_batch_result* result, int32_t cloud, int32_t k);
/* nclouds + 1 row offsets of diagram dim in the batch's rows of that dim
 * (cloud c's rows are [out[c], out[c+1]); all zero when no cloud has dim) */
int ph_batch_result_offsets(const ph_batch_result* result, int32_t dim, int64_t* out);
/* copies all rows of diagram dim (out[nclouds] x 2 float32) to dst, device or
 * host memory, on any stream (the run's frees wait for the copy) */
int ph_batch_result_copy(const ph_batch_result* result, int32_t dim, float* dst, int32_t to_host, void* stream);
/* releases the rows and the run's buffers (stream-ordered on the run's stream) */
void ph_batch_result_free(ph_batch_result* result);

/* ---- batches of clouds ---------------------------------------------------- */
/* The reference has no batched API; each entry below does, for every cloud of
 * a batch at once, what the cited per-cloud step does for one cloud. */

/* vcloud[v] = cloud of global vertex v (N = sum of n over the batch); batch
 * bookkeeping with no per-cloud counterpart. */
int ph_batch_vertex_cloud(const ph_cloud_seg* segs, int32_t nsegs, int32_t* vcloud, void* stream);

/* Per-cloud filtration order of a batch's edges: each cloud's edges sorted
 * by the reference's packed key computed with local vertex indices
 * (rips.py:30-50), clouds in batch order. any_wrap != 0 when some cloud has
 * n > 92682 (packed-key ties are then put in the reference's emission order). */
size_t ph_batch_edges_sort_workspace_bytes(int64_t E);
int ph_batch_edges_sort(const int32_t* in_i, const int32_t* in_j, const float* in_dsq, int64_t E,
                        const int32_t* vcloud, const ph_cloud_seg* segs, int32_t nsegs, int32_t any_wrap,
                        int32_t* out_i, int32_t* out_j, float* out_dsq, void* workspace,
                        size_t workspace_bytes, void* stream);

/* off[c] = first item of cloud c for items grouped by cloud, identified by
 * one vertex each (item_vertex); off[nsegs] = n_items. Batch bookkeeping
 * with no per-cloud counterpart. */
int ph_batch_item_offsets(const int32_t* item_vertex, int64_t n_items, const int32_t* vcloud, int32_t nsegs,
                          int64_t* off, void* stream);

/* H0 rows per cloud (persistence.py:169-192): cloud c's n rows start at row
 * vbase_c. edge_off: per-cloud edge offsets. out_rows: N x 2. */
size_t ph_batch_h0_rows_workspace_bytes(int64_t E);
int ph_batch_h0_rows(const float* edge_filt, const uint8_t* mst_mask, int64_t E, const int64_t* edge_off,
                     const ph_cloud_seg* segs, int32_t nsegs, const int32_t* vcloud, int64_t N,
                     float* out_rows, void* workspace, size_t workspace_bytes, void* stream);

/* ph_persistence_rows per cloud (reduce_h1_gpu.py:574-604 per cloud):
 * col_off (nsegs+1) are the per-cloud column offsets; row_off (nsegs+1)
 * receives the per-cloud row offsets. */
size_t ph_batch_persistence_rows_workspace_bytes(int64_t K);
int ph_batch_persistence_rows(const int32_t* col_state, const int32_t* col_piv, int64_t K, int32_t row_base,
                              const float* filt, const int32_t* col_m, const int32_t* row_m,
                              const int64_t* col_off, int32_t nsegs, float* out_rows, int64_t* row_off,
                              int64_t* d_nrows, void* workspace, size_t workspace_bytes, void* stream);

/* out[e] = 1 if edge e's cloud has max_dim >= min_dim: the per-cloud
 * max_dim branch of persistence.py:185-215 as an edge mask. */
int ph_batch_edge_dim_mask(const int32_t* edge_i, int64_t E, const int32_t* vcloud, const ph_cloud_seg* segs,
                           int32_t min_dim, uint8_t* out, void* stream);

/* dst[i] |= src[idx[i]] (or its negation when invert != 0); mask plumbing
 * for the batch, no per-cloud counterpart. */
int ph_or_gather_mask(uint8_t* dst, const uint8_t* src, const int32_t* idx, int64_t n, int32_t invert,
                      void* stream);

/* k-th nearest-neighbour distance of every point of every cloud, k clamped
 * to n_c - 1 per cloud (threshold.py:133-176 _tiled_knn per cloud). qb_off (nsegs+1): per-cloud offsets of 128-point
 * query blocks; nqb their total; max_d the largest d. out: N floats. */
int ph_batch_knn_kth(const float* pts, const ph_cloud_seg* segs, int32_t nsegs, const int64_t* qb_off,
                     int64_t nqb, int32_t max_d, int32_t k, float* out, void* stream);

/* torch.quantile semantics per cloud over values[vbase_c .. vbase_c+n_c)
 * (the quantile of threshold.py:77 per cloud). */
size_t ph_batch_quantile_workspace_bytes(int64_t N);
int ph_batch_quantile(const float* values, int64_t N, const int32_t* vcloud, const ph_cloud_seg* segs,
                      int32_t nsegs, double q, float* out, void* workspace, size_t workspace_bytes,
                      void* stream);

/* ---- thresholds ---------------------------------------------------------- */

/* k-th nearest-neighbour Euclidean distance of every point (self excluded),
 * threshold.py:133-176 _tiled_knn. k <= 64. out: n float32. */
int ph_knn_kth(const float* pts, int64_t n, int32_t d, int32_t k, float* out, void* stream);

/* Linear-interpolation quantile of n values (torch.quantile semantics, as
 * threshold.py:77 uses it); *d_out (float32, device). */
size_t ph_quantile_workspace_bytes(int64_t n);
int ph_quantile_f32(const float* values, int64_t n, double q, float* d_out, void* workspace,
                    size_t workspace_bytes, void* stream);

/* min over points of the max distance to any point, threshold.py:179-200
 * _tiled_enclosing_radius; *d_out (float32, device). */
size_t ph_enclosing_radius_workspace_bytes(int64_t n);
int ph_enclosing_radius(const float* pts, int64_t n, int32_t d, float* d_out, void* workspace,
                        size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLASHPH_B200_H_ */
