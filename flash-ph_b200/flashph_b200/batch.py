"""Batching form: many point clouds of uneven n and d in one pipeline.

A batch is the disjoint union of its clouds (vertex v of cloud c has global
index vbase_c + v). ``rips_persistence_batch`` runs it through one native
library call per chunk (``ph_rips_persistence_batch``): edge enumeration
walks (cloud, tile) work items from a segment table, the filtration sort
orders every cloud's edges by its own packed key (local indices), and
everything after it -- adjacency, forest, triangles, tetrahedra, cofacets,
the lock-free reduction -- runs on global indices unchanged, because no
simplex spans two clouds; the host waits four times per chunk, whatever the
number of clouds. Rows are cut per cloud at the end. Every cloud's diagrams
equal those of a separate ``rips_persistence`` call on it, bit for bit.

Clouds are processed in chunks bounded by points and pairs; a chunk whose
simplices exceed the rank range or the per-chunk simplex budget is split by
the exact per-cloud counts the library returns. Errors that the reference
raises per call (validation, the triangle and tetrahedron caps) are
returned per cloud as exception objects; they do not stop the batch.

``FLASHPH_BATCH=staged`` runs the same union stage by stage from Python
(each stage its own library call), a cross-check of the native call.
"""
from __future__ import annotations

import ctypes
import math
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import Sequence

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from .boruvka import boruvka_mask
from .cohomology import Reduction, cof_max_face, cofacet_csr, grow_pool, pool_capacity, reduce as _reduce
from .persistence import _compute_native
from .rips import edge_filtration_values, threshold_sq, vertex_csr

PH_ERR_POOL = 5
SEG_DTYPE = np.dtype([("pt_off", "<i8"), ("vbase", "<i8"), ("tile_off", "<i8"), ("n", "<i4"), ("d", "<i4"),
                      ("thr_sq", "<f4"), ("max_dim", "<i4")])
assert SEG_DTYPE.itemsize == 40

_CHUNK_POINTS = 1 << 18
_CHUNK_PAIRS = 1 << 34
_CHUNK_TRIANGLES = 1 << 28   # per chunk, keeps every global rank in int32
_CHUNK_TETS = 1 << 28
NATIVE_MIN_POINTS = 1024  # staged form only: clouds this large run as native single calls
_NATIVE_WORKERS = 2
# native batch chunks: points, candidate pairs and simplices (triangles, plus
# tetrahedra for H2) per library call
_BATCH_POINTS = 1 << 20
_BATCH_PAIRS = 1 << 36
_BATCH_SIMPLICES = 1 << 27
_EDGE_MODES = {"auto": 0, "on": 1, "off": 2}


# Worker streams are kept for the life of the process and reused (by the
# native workers below and by serve.py's slots): torch's caching allocator
# keeps its free blocks per stream, so fresh streams would start every call
# with cold caches (fresh device allocations, which can wait for the device).
_STREAMS: dict = {}
_STREAMS_LOCK = threading.Lock()


def worker_stream(device, index: int):
    key = (device.index if device.index is not None else torch.cuda.current_device(), index)
    with _STREAMS_LOCK:
        if key not in _STREAMS:
            _STREAMS[key] = torch.cuda.Stream(device)
        return _STREAMS[key]


def _run_native(items, device, max_triangles, max_tetrahedra):
    """(cloud, points, t, max_dim) items as native calls on worker streams;
    returns {cloud: diagrams or the reference's exception}."""
    caller = torch.cuda.current_stream(device)
    ready = torch.cuda.Event()
    ready.record(caller)  # inputs written on the caller's stream are complete before the workers read them
    local = threading.local()
    taken = iter(range(_NATIVE_WORKERS))
    taken_lock = threading.Lock()

    def one(item):
        c, p, t, md = item
        if not hasattr(local, "stream"):
            with taken_lock:
                idx = next(taken)
            local.stream = worker_stream(device, 100 + idx)  # indices apart from the server's slots
            local.stream.wait_event(ready)
        with torch.cuda.device(device), torch.cuda.stream(local.stream):
            try:
                x = p.to(device).float().contiguous()
                out = _compute_native(x, t, md, device, max_triangles, max_tetrahedra)
                for o in out:
                    o.record_stream(caller)  # the caller's later use keeps the memory from early reuse
            except ValueError as ex:  # the reference's per-call errors
                out = ex
        local.stream.synchronize()
        return c, out

    with ThreadPoolExecutor(max_workers=_NATIVE_WORKERS) as ex:
        return dict(ex.map(one, items))


def _validate(points, t, max_dim):
    if t < 0:
        return ValueError(f"max_edge_length must be non-negative, got {t}")
    if points.ndim != 2:
        return ValueError(f"points must have shape (n, d), got {tuple(points.shape)}")
    if max_dim not in (0, 1, 2):
        return ValueError(f"max_dim must be 0, 1, or 2, got {max_dim}")
    if max_dim == 2 and points.shape[0] >= (1 << 16):
        return ValueError(
            f"H2 requires n < 65536 (16-bit vertex packing), got n={points.shape[0]}. "
            f"Use max_dim=1 or reduce n.")
    return None


def _trivial(n, max_dim, device):
    e = lambda: torch.empty(0, 2, dtype=torch.float32, device=device)  # noqa: E731
    if n == 0:
        return [e() for _ in range(max_dim + 1)]
    h0 = torch.tensor([[0.0, float("inf")]], dtype=torch.float32, device=device)
    return [h0] + [e() for _ in range(max_dim)]


class _Batch:
    """Device-side layout of one chunk of clouds."""

    def __init__(self, pts_list, thrs, dims, device):
        self.device = device
        self.k = len(pts_list)
        segs = np.zeros(self.k, dtype=SEG_DTYPE)
        pt_off = vbase = tile_off = 0
        for c, (p, t, md) in enumerate(zip(pts_list, thrs, dims)):
            n, d = int(p.shape[0]), int(p.shape[1])
            segs[c] = (pt_off, vbase, tile_off, n, d, threshold_sq(t), md)
            pt_off += n * d
            vbase += n
            tile_off += int(L.query("ph_cloud_tiles", n))
        self.segs_np = segs
        self.N = vbase
        self.ntiles = tile_off
        self.max_dim = max(dims) if dims else 0
        self.any_wrap = int(any(int(p.shape[0]) > 92682 for p in pts_list))
        flat = [p.reshape(-1).float() for p in pts_list]
        if not flat:
            self.pts = torch.empty(0, device=device)
        elif all(f.device.type == "cpu" for f in flat):
            host = torch.cat(flat)
            self.pts = host.pin_memory().to(device, non_blocking=True) if host.numel() else host.to(device)
        else:
            self.pts = torch.cat([f.to(device) for f in flat])
        self.segs = torch.from_numpy(segs.view(np.uint8).copy()).to(device)
        self.vcloud = torch.empty(max(self.N, 1), dtype=torch.int32, device=device)
        L.call("ph_batch_vertex_cloud", self.segs.data_ptr(), self.k, self.vcloud.data_ptr(),
               L.stream_handle(device))


def _edges(b: _Batch):
    from ._edges import enumerate_segments

    dev = b.device
    s = L.stream_handle(dev)
    pairs = sum(int(n) * (int(n) - 1) // 2 for n in b.segs_np["n"])
    cap = int(min(pairs, max(1 << 20, 256 * b.N)))
    ei, ej, ed = enumerate_segments(b.pts, b.segs_np, b.segs, b.ntiles, cap)
    E = ei.numel()
    oi, oj, od = torch.empty_like(ei), torch.empty_like(ej), torch.empty_like(ed)
    if E:
        nb = L.query("ph_batch_edges_sort_workspace_bytes", E)
        ws = L.workspace(nb, dev)
        L.call("ph_batch_edges_sort", ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), E, b.vcloud.data_ptr(),
               b.segs.data_ptr(), b.k, b.any_wrap, oi.data_ptr(), oj.data_ptr(), od.data_ptr(), ws.data_ptr(),
               nb, s)
    return oi, oj, od


def _item_offsets(b: _Batch, item_vertex: Tensor):
    off = torch.empty(b.k + 1, dtype=torch.int64, device=b.device)
    L.call("ph_batch_item_offsets", L.ptr(item_vertex), item_vertex.numel(), b.vcloud.data_ptr(), b.k,
           off.data_ptr(), L.stream_handle(b.device))
    return off


def _rows(red: Reduction, K: int, row_base: int, filt: Tensor, col_m, row_m, col_off: Tensor, nsegs: int):
    dev = filt.device
    rows = torch.empty(max(K, 1), 2, dtype=torch.float32, device=dev)
    row_off = torch.empty(nsegs + 1, dtype=torch.int64, device=dev)
    nrows = torch.zeros(1, dtype=torch.int64, device=dev)
    nb = L.query("ph_batch_persistence_rows_workspace_bytes", K)
    ws = L.workspace(nb, dev)
    L.call("ph_batch_persistence_rows", L.ptr(red.state), L.ptr(red.piv), K, row_base, L.ptr(filt), L.ptr(col_m),
           L.ptr(row_m), col_off.data_ptr(), nsegs, rows.data_ptr(), row_off.data_ptr(), nrows.data_ptr(),
           ws.data_ptr(), nb, L.stream_handle(dev))
    return rows, row_off


class _Filt:
    """RipsFiltration-shaped record for the shared stage functions."""

    def __init__(self, ei, ej, ed, ptr, idx, rank):
        self.edge_i, self.edge_j, self.edge_dist_sq = ei, ej, ed
        self.vert_adj_ptr, self.vert_adj_idx, self.vert_adj_rank = ptr, idx, rank


def _run_chunk(pts_list, thrs, dims, device, max_triangles, max_tetrahedra):
    """Diagrams of every cloud of one chunk; raises _CapExceeded on caps."""
    from .cohomology import count_triangles, emit_triangles

    b = _Batch(pts_list, thrs, dims, device)
    dev = device
    s = L.stream_handle(dev)
    ei, ej, ed = _edges(b)
    E = ei.numel()
    ptr, idx, rank = vertex_csr(ei, ej, b.N)
    f = _Filt(ei, ej, ed, ptr, idx, rank)
    filt = edge_filtration_values(ed)
    mst, _, (_, mst_status) = boruvka_mask(ei, ej, b.N)
    e_off = _item_offsets(b, ei)
    h0 = torch.empty(max(b.N, 1), 2, dtype=torch.float32, device=dev)
    nb = L.query("ph_batch_h0_rows_workspace_bytes", E)
    ws = L.workspace(nb, dev)
    L.call("ph_batch_h0_rows", L.ptr(filt), L.ptr(mst), E, e_off.data_ptr(), b.segs.data_ptr(), b.k,
           b.vcloud.data_ptr(), b.N, h0.data_ptr(), ws.data_ptr(), nb, s)
    out = {"h0": h0, "h0_off": torch.from_numpy(b.segs_np["vbase"].astype(np.int64))}
    checks = [("ph_boruvka_mst", mst_status)]
    if b.max_dim >= 1:
        tri_off = count_triangles(f)
        t_per_cloud = (tri_off[e_off[1:]] - tri_off[e_off[:-1]]).cpu().numpy()
        over = [c for c in range(b.k) if dims[c] >= 1 and t_per_cloud[c] > max_triangles]
        if over:
            raise _CapExceeded({c: ValueError(
                f"Triangle count {int(t_per_cloud[c])} exceeds max_triangles={max_triangles}. "
                f"Reduce max_edge_length or increase max_triangles.") for c in over})
        T = int(t_per_cloud.sum())
        if E + 3 * T >= 2 ** 31 or T > _CHUNK_TRIANGLES:
            raise _ChunkTooBig()
        tris = emit_triangles(f, tri_off, T)
        if T:
            off1, data1 = cofacet_csr(E, E, T, 3, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb)
        else:
            off1 = torch.zeros(E + 1, dtype=torch.int32, device=dev)
            data1 = torch.empty(0, dtype=torch.int32, device=dev)
        # clouds that asked for H0 only get no H1 columns
        skip1 = mst.clone()
        if any(d < 1 for d in dims):
            m1 = torch.empty(max(E, 1), dtype=torch.uint8, device=dev)
            L.call("ph_batch_edge_dim_mask", L.ptr(ei), E, b.vcloud.data_ptr(), b.segs.data_ptr(), 1,
                   m1.data_ptr(), s)
            skip1 |= (m1[:E] == 0)
        cmf1 = cof_max_face(T, 3, 0, mst, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb)
        red1 = _reduce_retry(off1, data1, E, 0, T, E, skip1, cmf1, checks)
        h1, h1_off = _rows(red1, E, E, filt, None, tris.tri_m, e_off, b.k)
        out.update(h1=h1, h1_off=h1_off)
        if b.max_dim >= 2:
            en = torch.empty(max(E, 1), dtype=torch.uint8, device=dev)
            L.call("ph_batch_edge_dim_mask", L.ptr(ei), E, b.vcloud.data_ptr(), b.segs.data_ptr(), 2,
                   en.data_ptr(), s)
            en = en[:E] if E else en
            tet_off = torch.empty(E + 1, dtype=torch.int64, device=dev)
            nb = L.query("ph_tets_count_workspace_bytes", E)
            ws = L.workspace(nb, dev)
            L.call("ph_tets_count", tris.tri_off.data_ptr(), L.ptr(tris.tri_w), E, ptr.data_ptr(), L.ptr(idx),
                   L.ptr(rank), L.ptr(en), tet_off.data_ptr(), ws.data_ptr(), nb, s)
            q_per_cloud = (tet_off[e_off[1:]] - tet_off[e_off[:-1]]).cpu().numpy()
            over = [c for c in range(b.k) if dims[c] >= 2 and q_per_cloud[c] > max_tetrahedra]
            if over:
                raise _CapExceeded({c: ValueError(
                    f"Tetrahedra count {int(q_per_cloud[c])} exceeds max_tetrahedra={max_tetrahedra}. "
                    f"Reduce max_edge_length or increase max_tetrahedra.") for c in over})
            Q = int(q_per_cloud.sum())
            if E + T + Q >= 2 ** 31 or 4 * Q >= 2 ** 31 or Q > _CHUNK_TETS:
                raise _ChunkTooBig()
            tet_m = torch.empty(Q, dtype=torch.int32, device=dev)
            tet_f = torch.empty(4 * Q, dtype=torch.int32, device=dev)
            tstat = torch.zeros(1, dtype=torch.int32, device=dev)
            if Q:
                L.call("ph_tets_emit", L.ptr(ei), L.ptr(ej), E, tris.tri_off.data_ptr(), L.ptr(tris.tri_w),
                       L.ptr(tris.tri_fa), L.ptr(tris.tri_fb), ptr.data_ptr(), L.ptr(idx), L.ptr(rank), L.ptr(en),
                       tet_off.data_ptr(), tet_m.data_ptr(), tet_f.data_ptr(), tstat.data_ptr(), s)
            skip2 = torch.empty(max(T, 1), dtype=torch.uint8, device=dev)
            L.call("ph_mark_pivots", L.ptr(red1.state), L.ptr(red1.piv), E, E, skip2.data_ptr(), T, s)
            if T:  # triangles of clouds without H2 are not columns
                L.call("ph_or_gather_mask", skip2.data_ptr(), en.data_ptr(), tris.tri_m.data_ptr(), T, 1, s)
            cmf2 = cof_max_face(Q, 4, E, skip2, faces_aos=tet_f)
            if Q:
                off2, data2 = cofacet_csr(T, E + T, Q, 4, faces_aos=tet_f)
            else:
                off2 = torch.zeros(T + 1, dtype=torch.int32, device=dev)
                data2 = torch.empty(0, dtype=torch.int32, device=dev)
            checks.append(("ph_tets_emit", tstat))
            red2 = _reduce_retry(off2, data2, T, E, Q, E + T, skip2, cmf2, checks)
            t_off = tris.tri_off[e_off].contiguous()
            h2, h2_off = _rows(red2, T, E + T, filt, tris.tri_m, tet_m, t_off, b.k)
            out.update(h2=h2, h2_off=h2_off)
    # one host synchronisation for every status and offset
    parts = [st.long().reshape(-1) for _, st in checks]
    for key in ("h1_off", "h2_off"):
        if key in out:
            parts.append(out[key])
    host = torch.cat(parts).cpu() if parts else torch.empty(0)
    for k, (name, _) in enumerate(checks):
        if int(host[k]) != 0:
            raise L.PHError(name, int(host[k]))
    pos = len(checks)
    res = []
    off_h = {}
    for key in ("h1_off", "h2_off"):
        if key in out:
            off_h[key] = host[pos:pos + b.k + 1].tolist()
            pos += b.k + 1
    vb = b.segs_np["vbase"]
    for c in range(b.k):
        n = int(b.segs_np["n"][c])
        dg = [out["h0"][int(vb[c]): int(vb[c]) + n]]
        if dims[c] >= 1:
            o = off_h["h1_off"]
            dg.append(out["h1"][o[c]: o[c + 1]])
        if dims[c] >= 2:
            o = off_h["h2_off"]
            dg.append(out["h2"][o[c]: o[c + 1]])
        res.append(dg)
    return res


def _reduce_retry(off, data, K, col_base, R, row_base, skip, cmf, checks):
    """Reduction whose status is read with the final synchronisation; a pool
    overflow (rare) is detected here by a synchronous check and retried."""
    pool_cap = pool_capacity(int(data.numel()), K)
    for _ in range(4):
        red = _reduce(off, data, K, col_base, R, row_base, skip, cmf, pool_cap)
        st = int(red.status.item())
        if st == 0:
            return red
        if st != PH_ERR_POOL:
            raise L.PHError("ph_reduce", st)
        pool_cap = grow_pool(pool_cap)
    raise L.PHError("ph_reduce", PH_ERR_POOL, "pool still too small after retries")


class _ChunkTooBig(Exception):
    """The chunk's simplices do not fit the rank range or the memory budget."""


class _CapExceeded(Exception):
    def __init__(self, errors: dict):
        super().__init__("cap exceeded")
        self.errors = errors


def _chunks(order, sizes, max_points=_CHUNK_POINTS, max_pairs=_CHUNK_PAIRS):
    chunk, pts, pairs = [], 0, 0
    for c in order:
        n = sizes[c]
        if chunk and (pts + n > max_points or pairs + n * n // 2 > max_pairs):
            yield chunk
            chunk, pts, pairs = [], 0, 0
        chunk.append(c)
        pts += n
        pairs += n * n // 2
    if chunk:
        yield chunk


class _Split(Exception):
    """The chunk is over the rank range or the simplex budget; per-cloud
    simplex counts (triangles + tetrahedra where counted) come with it."""

    def __init__(self, counts: list[int], edges: list[int]):
        super().__init__("split")
        self.counts = counts
        self.edges = edges


def _native_chunk(pts: list[Tensor], ts: list[float], dims: list[int], device, max_triangles: int,
                  max_tetrahedra: int) -> list:
    """Diagrams (or the reference's ValueError) of every cloud of a chunk,
    from one ph_rips_persistence_batch call; raises _Split when the library
    asks for a smaller chunk."""
    lib = L.lib()
    k = len(pts)
    ptrs = (ctypes.c_void_p * k)(*[p.data_ptr() for p in pts])
    n = np.array([p.shape[0] for p in pts], dtype=np.int64)
    d = np.array([p.shape[1] for p in pts], dtype=np.int32)
    t = np.array(ts, dtype=np.float64)
    md = np.array(dims, dtype=np.int32)
    mode = _edge_mode(pts, ts, n, d, device)
    s = L.stream_handle(device)
    res = ctypes.c_void_p()
    rc = lib.ph_rips_persistence_batch(ptrs, n.ctypes.data, d.ctypes.data, t.ctypes.data, md.ctypes.data, k,
                                       max_triangles, max_tetrahedra, mode, _BATCH_SIMPLICES, ctypes.byref(res), s)
    if rc == 3 and res.value:  # PH_ERR_CAPACITY: split by the exact counts
        try:
            tri = [max(0, int(lib.ph_batch_result_stat(res, c, 1))) for c in range(k)]
            tet = [max(0, int(lib.ph_batch_result_stat(res, c, 2))) for c in range(k)]
            edg = [max(0, int(lib.ph_batch_result_stat(res, c, 0))) for c in range(k)]
        finally:
            lib.ph_batch_result_free(res)
        raise _Split([a + b for a, b in zip(tri, tet)], edg)
    if rc != L.PH_OK:
        raise L.PHError("ph_rips_persistence_batch", rc, lib.ph_last_error().decode(errors="replace"))
    try:
        top = max(dims)
        bufs, offs = [], []
        for dim in range(top + 1):
            off = np.zeros(k + 1, dtype=np.int64)
            L.call("ph_batch_result_offsets", res, dim, off.ctypes.data)
            buf = torch.empty(max(int(off[-1]), 1), 2, dtype=torch.float32, device=device)
            L.call("ph_batch_result_copy", res, dim, buf.data_ptr(), 0, s)
            bufs.append(buf)
            offs.append(off)
        out = []
        for c in range(k):
            if int(lib.ph_batch_result_status(res, c)) != L.PH_OK:
                out.append(ValueError(lib.ph_batch_result_message(res, c).decode(errors="replace")))
                continue
            out.append([bufs[dim][int(offs[dim][c]):int(offs[dim][c + 1])] for dim in range(dims[c] + 1)])
    finally:
        lib.ph_batch_result_free(res)
    return out


def _edge_mode(pts: list[Tensor], ts: list[float], n: np.ndarray, d: np.ndarray, device) -> int:
    """The chunk's edge kernel: FLASHPH_EDGE_SCREEN=on / off, else the
    autotuner's choice for the chunk's (largest d, mean cloud size) key (one
    timed trial of both kernels on the first chunk of each key)."""
    env = os.environ.get("FLASHPH_EDGE_SCREEN", "auto").lower()
    if env in ("on", "off"):
        return _EDGE_MODES[env]
    from . import autotune
    from ._edges import enumerate_segments

    key_segs = np.zeros(len(pts), dtype=SEG_DTYPE)
    key_segs["n"] = n
    key_segs["d"] = d
    state = {}

    def trial(screen: bool) -> int:
        if "b" not in state:  # the chunk's union layout, built only when a trial runs
            state["b"] = _Batch(pts, ts, [0] * len(pts), device)
        b = state["b"]
        pairs = sum(int(x) * (int(x) - 1) // 2 for x in n)
        cap = int(min(pairs, max(1 << 20, 256 * b.N)))
        ei, _, _ = enumerate_segments(b.pts, b.segs_np, b.segs, b.ntiles, cap, screen=screen)
        return int(ei.numel())

    return autotune.choose(key_segs, trial)


def _repack(chunk: list[int], counts: list[int], edges: list[int]) -> list[list[int]]:
    """A split chunk packed again by its exact per-cloud simplex counts."""
    parts, cur, simp, ed = [], [], 0, 0
    for c, q, e in zip(chunk, counts, edges):
        if cur and (simp + q > _BATCH_SIMPLICES or ed + e + 3 * (simp + q) >= (1 << 31) - (1 << 24)):
            parts.append(cur)
            cur, simp, ed = [], 0, 0
        cur.append(c)
        simp += q
        ed += e
    if cur:
        parts.append(cur)
    if len(parts) == 1 and len(chunk) > 1:  # the counts fit after all (the budget counts H2 too): halve
        h = len(chunk) // 2
        parts = [chunk[:h], chunk[h:]]
    return parts


def _to_device_all(pts: list[Tensor], device) -> list[Tensor]:
    """float32 contiguous device copies of the clouds; host clouds go over in
    one pinned copy."""
    host = [i for i, p in enumerate(pts) if p.device.type != "cuda"]
    out = list(pts)
    if host:
        flat = torch.cat([pts[i].reshape(-1).float() for i in host])
        dev = flat.pin_memory().to(device, non_blocking=True) if flat.numel() else flat.to(device)
        at = 0
        for i in host:
            m = pts[i].numel()
            out[i] = dev[at:at + m].view(pts[i].shape[0], pts[i].shape[1])
            at += m
    for i, p in enumerate(out):
        if i not in host:
            out[i] = p.to(device).float().contiguous()
    return out


def rips_persistence_batch(
    clouds: Sequence,
    max_edge_lengths,
    max_dim=1,
    max_triangles: int = 10_000_000,
    max_tetrahedra: int = 10_000_000,
):
    """Persistence diagrams of many point clouds.

    Parameters
    ----------
    clouds : sequence of (n_c, d_c) arrays or tensors (n and d may differ).
    max_edge_lengths : float or sequence of floats, one per cloud.
    max_dim : int or sequence of ints (0, 1 or 2), one per cloud.
    max_triangles, max_tetrahedra : per-cloud caps (the reference's defaults).

    Returns
    -------
    list, one entry per cloud: the list of diagrams ``rips_persistence``
    returns for that cloud (on the CUDA device), or the exception the
    reference would raise for it.
    """
    k = len(clouds)
    ts = [float(max_edge_lengths)] * k if np.isscalar(max_edge_lengths) else [float(x) for x in max_edge_lengths]
    ds = [int(max_dim)] * k if np.isscalar(max_dim) else [int(x) for x in max_dim]
    if len(ts) != k or len(ds) != k:
        raise ValueError("one max_edge_length and one max_dim per cloud")
    if not torch.cuda.is_available():
        raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
    device = torch.device("cuda", torch.cuda.current_device())
    pts, results, todo = [], [None] * k, []
    for c, p in enumerate(clouds):
        t = p if isinstance(p, Tensor) else torch.from_numpy(np.ascontiguousarray(p))
        err = _validate(t, ts[c], ds[c])
        pts.append(t)
        if err is not None:
            results[c] = err
        elif t.shape[0] <= 1:
            results[c] = _trivial(t.shape[0], ds[c], device)
        else:
            todo.append(c)
    if os.environ.get("FLASHPH_BATCH", "native") == "staged":
        _staged_batch(pts, ts, ds, todo, results, device, max_triangles, max_tetrahedra)
        return results
    dev_pts = _to_device_all([pts[c] for c in todo], device)
    dpts = dict(zip(todo, dev_pts))
    sizes = {c: int(pts[c].shape[0]) for c in todo}
    work = list(_chunks(todo, sizes, _BATCH_POINTS, _BATCH_PAIRS))
    while work:
        chunk = work.pop(0)
        try:
            res = _native_chunk([dpts[c] for c in chunk], [ts[c] for c in chunk], [ds[c] for c in chunk], device,
                                max_triangles, max_tetrahedra)
        except _Split as sp:
            if len(chunk) == 1:  # one cloud beyond the int32 rank range
                results[chunk[0]] = ValueError("Simplex count exceeds the int32 rank range")
                continue
            work[:0] = _repack(chunk, sp.counts, sp.edges)
            continue
        for c, r in zip(chunk, res):
            results[c] = r
    return results


def _staged_batch(pts, ts, ds, todo, results, device, max_triangles, max_tetrahedra):
    """The union stage by stage from Python (cross-check of the native batch)."""
    native = [c for c in todo if int(pts[c].shape[0]) >= NATIVE_MIN_POINTS]
    if native:
        done = _run_native([(c, pts[c], ts[c], ds[c]) for c in native], device, max_triangles, max_tetrahedra)
        for c, r in done.items():
            results[c] = r
        todo = [c for c in todo if int(pts[c].shape[0]) < NATIVE_MIN_POINTS]
    sizes = {c: int(pts[c].shape[0]) for c in todo}
    work = list(_chunks(todo, sizes))
    while work:
        chunk = work.pop(0)
        try:
            res = _run_chunk([pts[c].float().contiguous() for c in chunk], [ts[c] for c in chunk],
                             [ds[c] for c in chunk], device, max_triangles, max_tetrahedra)
            for c, r in zip(chunk, res):
                results[c] = r
        except _CapExceeded as ex:
            for local, err in ex.errors.items():
                results[chunk[local]] = err
            rest = [c for i, c in enumerate(chunk) if i not in ex.errors]
            if rest:
                work.insert(0, rest)
        except _ChunkTooBig:
            if len(chunk) == 1:
                results[chunk[0]] = ValueError("Simplex count exceeds the int32 rank range")
            else:
                h = len(chunk) // 2
                work[:0] = [chunk[:h], chunk[h:]]


def auto_threshold_batch(clouds: Sequence, k: int = 20, percentile: float = 95.0) -> list[float]:
    """``auto_threshold`` of every cloud (threshold.py:20-78), in one pass."""
    if not torch.cuda.is_available():
        raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
    device = torch.device("cuda", torch.cuda.current_device())
    pts = [p if isinstance(p, Tensor) else torch.from_numpy(np.ascontiguousarray(p)) for p in clouds]
    out = [0.0] * len(pts)
    live = [c for c, p in enumerate(pts) if p.shape[0] > 1]
    if not live:
        return out
    pct = max(0.0, min(100.0, percentile))
    b = _Batch([pts[c].float().contiguous() for c in live], [0.0] * len(live), [0] * len(live), device)
    qb = np.zeros(b.k + 1, dtype=np.int64)
    qb[1:] = np.cumsum((b.segs_np["n"].astype(np.int64) + 127) // 128)
    qb_dev = torch.from_numpy(qb).to(device)
    kth = torch.empty(max(b.N, 1), dtype=torch.float32, device=device)
    s = L.stream_handle(device)
    L.call("ph_batch_knn_kth", b.pts.data_ptr(), b.segs.data_ptr(), b.k, qb_dev.data_ptr(), int(qb[-1]),
           int(b.segs_np["d"].max()), max(1, k), kth.data_ptr(), s)
    res = torch.empty(b.k, dtype=torch.float32, device=device)
    nb = L.query("ph_batch_quantile_workspace_bytes", b.N)
    ws = L.workspace(nb, device)
    L.call("ph_batch_quantile", kth.data_ptr(), b.N, b.vcloud.data_ptr(), b.segs.data_ptr(), b.k, pct / 100.0,
           res.data_ptr(), ws.data_ptr(), nb, s)
    vals = res.cpu().tolist()
    for c, v in zip(live, vals):
        out[c] = float(v)
    return out
