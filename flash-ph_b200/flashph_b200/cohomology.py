"""H1 and H2 by cohomology on the GPU.

Reference: reduce_h1_gpu.py:438-604 (H1 pipeline) and, for H2, the
reference's building blocks (triangle_kernel.py:402 tetrahedra,
apparent_pair_h2_kernel.py, cohomology_general.py:32-199,622-701) that its
public path replaces with giotto-ph.

Columns are the simplices of one dimension in filtration order, rows the
simplices one dimension up: H1 columns are edges (global rank = edge rank),
rows are triangles (global rank E + position); H2 columns are triangles,
rows tetrahedra (global rank E + T + position). H2 columns that are H1
pivots are cleared (skipped), as in cohomology_general.py:635.
"""
from __future__ import annotations

from typing import NamedTuple

import torch
from torch import Tensor

from . import _lib as L
from . import _timing

PH_ERR_POOL = 5
_MAX_POOL_RETRIES = 4


class Triangles(NamedTuple):
    T: int
    tri_off: Tensor  # (E+1,) int64: triangles with largest edge m are [tri_off[m], tri_off[m+1])
    tri_m: Tensor    # (T,) int32 largest edge
    tri_w: Tensor    # (T,) int32 third vertex
    tri_fa: Tensor   # (T,) int32 rank of edge (a, w)
    tri_fb: Tensor   # (T,) int32 rank of edge (b, w)


class Reduction(NamedTuple):
    state: Tensor   # (K,) int32: 0 skipped, 1 apparent, 2 paired, 3 essential
    piv: Tensor     # (K,) int32 pivot global rank or -1
    info: Tensor    # (4,) int64 [residual columns, column additions, pool entries used, takeovers]
    status: Tensor  # (1,) int32 device status


def count_triangles(filt) -> Tensor:
    """tri_off (E+1, int64): triangles grouped by largest edge (no host sync)."""
    dev = filt.edge_i.device
    E = filt.edge_i.shape[0]
    tri_off = torch.empty(E + 1, dtype=torch.int64, device=dev)
    cof_off = torch.empty(E + 1, dtype=torch.int64, device=dev)
    nb = L.query("ph_triangles_count_workspace_bytes", E)
    ws = L.workspace(nb, dev)
    L.call("ph_triangles_count", L.ptr(filt.edge_i), L.ptr(filt.edge_j), E, filt.vert_adj_ptr.data_ptr(),
           L.ptr(filt.vert_adj_idx), L.ptr(filt.vert_adj_rank), tri_off.data_ptr(), cof_off.data_ptr(),
           ws.data_ptr(), nb, L.stream_handle(dev))
    return tri_off


def emit_triangles(filt, tri_off: Tensor, T: int) -> Triangles:
    dev = filt.edge_i.device
    E = filt.edge_i.shape[0]
    tm = torch.empty(T, dtype=torch.int32, device=dev)
    tw = torch.empty(T, dtype=torch.int32, device=dev)
    tfa = torch.empty(T, dtype=torch.int32, device=dev)
    tfb = torch.empty(T, dtype=torch.int32, device=dev)
    if T:
        L.call("ph_triangles_emit", L.ptr(filt.edge_i), L.ptr(filt.edge_j), E, filt.vert_adj_ptr.data_ptr(),
               L.ptr(filt.vert_adj_idx), L.ptr(filt.vert_adj_rank), tri_off.data_ptr(), tm.data_ptr(),
               tw.data_ptr(), tfa.data_ptr(), tfb.data_ptr(), L.stream_handle(dev))
    return Triangles(T, tri_off, tm, tw, tfa, tfb)


def enumerate_triangles(filt, max_triangles: int = 10_000_000) -> Triangles:
    E = filt.edge_i.shape[0]
    tri_off = count_triangles(filt)
    T = int(tri_off[E].item())
    if T > max_triangles:
        raise ValueError(
            f"Triangle count {T} exceeds max_triangles={max_triangles}. "
            f"Reduce max_edge_length or increase max_triangles.")
    if E + 3 * T >= 2 ** 31:
        raise ValueError(f"Triangle count {T} exceeds the int32 rank range")
    return emit_triangles(filt, tri_off, T)


def cofacet_csr(n_faces: int, row_base: int, S: int, k: int, faces_aos=None, f0=None, f1=None, f2=None):
    dev = (faces_aos if faces_aos is not None else f0).device
    off = torch.empty(n_faces + 1, dtype=torch.int32, device=dev)
    data = torch.empty(S * k, dtype=torch.int32, device=dev)
    nb = L.query("ph_cofacet_csr_workspace_bytes", S, k)
    ws = L.workspace(nb, dev)
    L.call("ph_cofacet_csr", L.ptr(faces_aos), L.ptr(f0), L.ptr(f1), L.ptr(f2), k, S, n_faces, row_base,
           off.data_ptr(), L.ptr(data), ws.data_ptr(), nb, L.stream_handle(dev))
    return off, data


def cof_max_face(S: int, k: int, face_base: int, skip: Tensor, faces_aos=None, f0=None, f1=None, f2=None):
    dev = skip.device
    cmf = torch.empty(S, dtype=torch.int32, device=dev)
    if S:
        L.call("ph_cof_max_face", L.ptr(faces_aos), L.ptr(f0), L.ptr(f1), L.ptr(f2), k, S, face_base,
               L.ptr(skip), cmf.data_ptr(), L.stream_handle(dev))
    return cmf


def reduce(cof_off: Tensor, cof_data: Tensor, K: int, col_base: int, R: int, row_base: int,
           skip: Tensor | None, cmf: Tensor, pool_cap: int, span: int = 0) -> Reduction:
    """Enqueue the reduction (no host synchronisation). ``span``: the most
    rows one column's entries can span (0: all R rows)."""
    dev = cof_off.device
    state = torch.empty(K, dtype=torch.int32, device=dev)
    piv = torch.empty(K, dtype=torch.int32, device=dev)
    info = torch.zeros(4, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    pool = torch.empty(max(pool_cap, 1), dtype=torch.int32, device=dev)
    nb = L.query("ph_reduce_workspace_bytes", K, R, span)
    ws = L.workspace(nb, dev)
    L.call("ph_reduce", cof_off.data_ptr(), L.ptr(cof_data), K, col_base, R, row_base, span, L.ptr(skip),
           L.ptr(cmf), L.ptr(state), L.ptr(piv), pool.data_ptr(), pool_cap, info.data_ptr(),
           status.data_ptr(), ws.data_ptr(), nb, L.stream_handle(dev))
    return Reduction(state, piv, info, status)


def persistence_rows(red: Reduction, K: int, row_base: int, filt: Tensor, col_m, row_m):
    dev = filt.device
    rows = torch.empty(max(K, 1), 2, dtype=torch.float32, device=dev)
    nrows = torch.zeros(1, dtype=torch.int64, device=dev)
    nb = L.query("ph_persistence_rows_workspace_bytes", K)
    ws = L.workspace(nb, dev)
    L.call("ph_persistence_rows", L.ptr(red.state), L.ptr(red.piv), K, row_base, L.ptr(filt), L.ptr(col_m),
           L.ptr(row_m), rows.data_ptr(), nrows.data_ptr(), ws.data_ptr(), nb, L.stream_handle(dev))
    return rows, nrows


# record offsets in the reducer's owner words have 33 bits
_POOL_MAX = (1 << 33) - 1


def pool_capacity(nnz: int, K: int) -> int:
    """Initial reduction pool (int32 entries): the initial records (at most
    2 nnz), per-warp chunks and the reduced columns; generous for small
    problems, where a retry would cost more than the memory, and bounded by
    the record-offset range."""
    mult = 8 if nnz < (1 << 24) else 3
    return min(mult * nnz + 2 * K + (1 << 23), _POOL_MAX)


def grow_pool(cap: int) -> int:
    if cap >= _POOL_MAX:
        raise L.PHError("ph_reduce", PH_ERR_POOL, "pool at its maximum size")
    return min(cap * 4, _POOL_MAX)


def _reduce_to_rows(cof_off, cof_data, K, col_base, R, row_base, skip, cmf, filt, col_m, row_m,
                    checks=()):
    """Reduction + rows with one host synchronisation; grows the pool on demand.

    ``checks``: (entry point name, device status tensor) pairs of earlier
    stages, read back in the same copy and raised if non-zero.
    """
    pool_cap = pool_capacity(int(cof_data.numel()), K)
    for _ in range(_MAX_POOL_RETRIES):
        red = reduce(cof_off, cof_data, K, col_base, R, row_base, skip, cmf, pool_cap)
        rows, nrows = persistence_rows(red, K, row_base, filt, col_m, row_m)
        parts = [red.status.long(), nrows, red.info] + [st.long() for _, st in checks]
        host = torch.cat(parts).cpu()
        for k, (name, _) in enumerate(checks):
            if int(host[6 + k]) != 0:
                raise L.PHError(name, int(host[6 + k]))
        st = int(host[0])
        if st == 0:
            return rows[: int(host[1])], red, host[2:6]
        if st != PH_ERR_POOL:
            raise L.PHError("ph_reduce", st)
        pool_cap = grow_pool(pool_cap)
    raise L.PHError("ph_reduce", PH_ERR_POOL, "pool still too small after retries")


def h1_diagram(filt, edge_filt: Tensor, mst_mask: Tensor, max_triangles: int = 10_000_000, checks=()):
    """H1 rows in the reference's order, plus what H2 needs."""
    E = filt.edge_i.shape[0]
    with _timing.stage("h1.triangles"):
        tris = enumerate_triangles(filt, max_triangles)
    T = tris.T
    with _timing.stage("h1.cofacets"):
        off, data = cofacet_csr(E, E, T, 3, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb) if T else (
            torch.zeros(E + 1, dtype=torch.int32, device=edge_filt.device),
            torch.empty(0, dtype=torch.int32, device=edge_filt.device))
        cmf = cof_max_face(T, 3, 0, mst_mask, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb)
    with _timing.stage("h1.reduce"):
        rows, red, info = _reduce_to_rows(off, data, E, 0, T, E, mst_mask, cmf, edge_filt, None, tris.tri_m,
                                          checks=checks)
    return rows, tris, red, info


def h2_diagram(filt, edge_filt: Tensor, tris: Triangles, h1: Reduction, max_tetrahedra: int = 10_000_000,
               edge_enable: Tensor | None = None):
    dev = edge_filt.device
    E = filt.edge_i.shape[0]
    T = tris.T
    s = L.stream_handle(dev)
    tet_off = torch.empty(E + 1, dtype=torch.int64, device=dev)
    nb = L.query("ph_tets_count_workspace_bytes", E)
    ws = L.workspace(nb, dev)
    L.call("ph_tets_count", tris.tri_off.data_ptr(), L.ptr(tris.tri_w), E, filt.vert_adj_ptr.data_ptr(),
           L.ptr(filt.vert_adj_idx), L.ptr(filt.vert_adj_rank), L.ptr(edge_enable), tet_off.data_ptr(),
           ws.data_ptr(), nb, s)
    Q = int(tet_off[E].item())
    if Q > max_tetrahedra:
        raise ValueError(
            f"Tetrahedra count {Q} exceeds max_tetrahedra={max_tetrahedra}. "
            f"Reduce max_edge_length or increase max_tetrahedra.")
    if E + T + Q >= 2 ** 31 or 4 * Q >= 2 ** 31:
        raise ValueError(f"Tetrahedra count {Q} exceeds the int32 rank range")
    tet_m = torch.empty(Q, dtype=torch.int32, device=dev)
    tet_faces = torch.empty(Q * 4, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if Q:
        L.call("ph_tets_emit", L.ptr(filt.edge_i), L.ptr(filt.edge_j), E, tris.tri_off.data_ptr(),
               L.ptr(tris.tri_w), L.ptr(tris.tri_fa), L.ptr(tris.tri_fb), filt.vert_adj_ptr.data_ptr(),
               L.ptr(filt.vert_adj_idx), L.ptr(filt.vert_adj_rank), L.ptr(edge_enable), tet_off.data_ptr(),
               tet_m.data_ptr(), tet_faces.data_ptr(), status.data_ptr(), s)
    skip2 = torch.empty(max(T, 1), dtype=torch.uint8, device=dev)
    L.call("ph_mark_pivots", L.ptr(h1.state), L.ptr(h1.piv), E, E, skip2.data_ptr(), T, s)
    cmf2 = cof_max_face(Q, 4, E, skip2, faces_aos=tet_faces)
    if Q:
        off2, data2 = cofacet_csr(T, E + T, Q, 4, faces_aos=tet_faces)
    else:
        off2 = torch.zeros(T + 1, dtype=torch.int32, device=dev)
        data2 = torch.empty(0, dtype=torch.int32, device=dev)
    rows, red, info = _reduce_to_rows(off2, data2, T, E, Q, E + T, skip2, cmf2, edge_filt, tris.tri_m, tet_m,
                                      checks=[("ph_tets_emit", status)])
    return rows, red, info, Q
