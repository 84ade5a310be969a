"""Python handle on the CPU oracle (test infrastructure only).

The oracle (``ph_oracle.cpp``) restates the reference implementation's
algorithm on the CPU. Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, always as the checker or as the
timed CPU baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libph_oracle.so")

_lib = None
_DT = {1: np.int32, 2: np.int64, 3: np.float32}
ARRAYS = ("edge_i", "edge_j", "edge_dsq", "mst_idx", "h0", "tri_max_rank_sorted",
          "ap_births", "ap_deaths", "res_births", "res_deaths", "ess_births",
          "h1_all_pivots", "h1", "h2", "h2_births", "h2_deaths", "h2_ess", "slot_seq", "slot_rounds")
SCALARS = ("E", "n_components", "T", "Q", "cofacet_nnz", "n_apparent", "residual", "xor_ops",
           "xor_max", "xor_elems", "crit_path", "col_max", "E_full", "collapse_removed",
           "collapse_delayed", "collapse_rounds")


def build(force: bool = False) -> str:
    """Compile the oracle with make (a no-op when it is up to date)."""
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "ph_oracle.cpp"))):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.oracle_run.restype = ctypes.c_void_p
        lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_int64]
        lib.oracle_run_collapsed.restype = ctypes.c_void_p
        lib.oracle_run_collapsed.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int]
        lib.oracle_collapse_slots.restype = ctypes.c_void_p
        lib.oracle_collapse_slots.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_int]
        lib.oracle_edge_dsq.restype = None
        lib.oracle_edge_dsq.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p]
        lib.oracle_row_edges.restype = ctypes.c_void_p
        lib.oracle_row_edges.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        lib.oracle_run_edges.restype = ctypes.c_void_p
        lib.oracle_run_edges.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                         ctypes.c_int64, ctypes.c_int]
        lib.oracle_error.restype = ctypes.c_char_p
        lib.oracle_error.argtypes = [ctypes.c_void_p]
        lib.oracle_free.argtypes = [ctypes.c_void_p]
        lib.oracle_get.restype = ctypes.c_void_p
        lib.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                   ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
        lib.oracle_scalar.restype = ctypes.c_int64
        lib.oracle_scalar.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.oracle_threshold_sq.restype = ctypes.c_float
        lib.oracle_threshold_sq.argtypes = [ctypes.c_double]
        _lib = lib
    return _lib


def threshold_sq(max_edge_length: float) -> np.float32:
    return np.float32(_load().oracle_threshold_sq(float(max_edge_length)))


def run(points, max_edge_length: float, max_dim: int = 1, fused: bool = True,
        nthreads: int = 0, stop_after: int = 0, edge_filt=None) -> dict:
    """Run the oracle pipeline; returns a dict of numpy arrays and ints.

    ``fused=True`` accumulates dist^2 with a fused multiply-add per
    dimension (the compiled GPU kernel's arithmetic); ``fused=False`` uses a
    separate multiply and add (the reference kernel under the Triton
    interpreter). ``stop_after``: 0 everything, 1 filtration only, 2 through H0.
    ``edge_filt``: optional filtration value per sorted edge, used instead of
    the correctly rounded square root of dist^2.
    """
    lib = _load()
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    if pts.ndim != 2:
        raise ValueError("points must be (n, d)")
    n, d = pts.shape
    ov = None if edge_filt is None else np.ascontiguousarray(edge_filt, dtype=np.float32)
    h = lib.oracle_run(pts.ctypes.data if n else None, n, d, float(max_edge_length),
                       int(max_dim), int(bool(fused)), int(nthreads), int(stop_after),
                       None if ov is None or ov.size == 0 else ov.ctypes.data,
                       -1 if ov is None else ov.size)
    return _collect(lib, h)


def run_collapsed(points, max_edge_length: float, max_dim: int = 2, fused: bool = True,
                  nthreads: int = 0, relaxed: bool = False) -> dict:
    """The oracle pipeline on the edge-collapsed flag filtration (the step
    giotto-ph takes before its reduction in the reference's H2 path,
    persistence.py:48-51). Same keys as ``run``; ``edge_i``/``edge_j`` are
    the collapsed filtration's edges, ``E_full`` the uncollapsed edge count,
    ``collapse_removed``/``collapse_delayed`` what the collapse did.
    ``relaxed`` selects the round form with reservations (``collapse_rounds``
    rounds) instead of the last-to-first order. Small inputs only (n <= 4096)."""
    lib = _load()
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    if pts.ndim != 2:
        raise ValueError("points must be (n, d)")
    n, d = pts.shape
    h = lib.oracle_run_collapsed(pts.ctypes.data if n else None, n, d, float(max_edge_length),
                                 int(max_dim), int(bool(fused)), int(nthreads), int(bool(relaxed)))
    return _collect(lib, h)


def collapse_slots(points, max_edge_length: float, fused: bool = True, nthreads: int = 0) -> dict:
    """The edge collapse's slot per sorted edge computed two ways: last to
    first (``slot_seq``) and in dependency rounds (``slot_rounds``, with
    ``collapse_rounds`` rounds). A slot is the edge index from which the edge
    is present after the collapse, -1 when it is dropped. Small inputs only."""
    lib = _load()
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    if pts.ndim != 2:
        raise ValueError("points must be (n, d)")
    n, d = pts.shape
    h = lib.oracle_collapse_slots(pts.ctypes.data if n else None, n, d, float(max_edge_length),
                                  int(bool(fused)), int(nthreads))
    return _collect(lib, h)


def edge_dsq(points, edge_i, edge_j, fused: bool = True, nthreads: int = 0) -> np.ndarray:
    """dist^2 of the given pairs with the edge kernel's chain (edge_kernel.py:111-123)."""
    lib = _load()
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    ei = np.ascontiguousarray(edge_i, dtype=np.int32)
    ej = np.ascontiguousarray(edge_j, dtype=np.int32)
    out = np.empty(ei.shape[0], dtype=np.float32)
    if ei.shape[0]:
        lib.oracle_edge_dsq(pts.ctypes.data, pts.shape[0], pts.shape[1], ei.ctypes.data, ej.ctypes.data,
                            ei.shape[0], int(bool(fused)), int(nthreads), out.ctypes.data)
    return out


def row_edges(points, max_edge_length: float, rows, fused: bool = True, nthreads: int = 0) -> dict:
    """The edges (min, max) incident to each listed row, j ascending per row
    (keys edge_i, edge_j, edge_dsq): the rows' slice of the edge set."""
    lib = _load()
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float32))
    r = np.ascontiguousarray(rows, dtype=np.int32)
    h = lib.oracle_row_edges(pts.ctypes.data, pts.shape[0], pts.shape[1], float(max_edge_length),
                             r.ctypes.data, r.shape[0], int(bool(fused)), int(nthreads))
    return _collect(lib, h)


def run_edges(edge_i, edge_j, edge_dsq, n: int, max_dim: int = 1) -> dict:
    """The oracle pipeline from a given edge list in any order: emission order
    restored from (i, j), packed-key stable sort, H0..H2 (keys as ``run``)."""
    lib = _load()
    ei = np.ascontiguousarray(edge_i, dtype=np.int32)
    ej = np.ascontiguousarray(edge_j, dtype=np.int32)
    ed = np.ascontiguousarray(edge_dsq, dtype=np.float32)
    E = ei.shape[0]
    h = lib.oracle_run_edges(ei.ctypes.data if E else None, ej.ctypes.data if E else None,
                             ed.ctypes.data if E else None, E, int(n), int(max_dim))
    return _collect(lib, h)


def _collect(lib, h) -> dict:
    try:
        err = lib.oracle_error(h)
        if err:
            raise ValueError(err.decode())
        out = {}
        for name in ARRAYS:
            cnt = ctypes.c_int64()
            dt = ctypes.c_int()
            ptr = lib.oracle_get(h, name.encode(), ctypes.byref(cnt), ctypes.byref(dt))
            dtype = _DT[dt.value]
            if cnt.value > 0:
                buf = (ctypes.c_char * (cnt.value * np.dtype(dtype).itemsize)).from_address(ptr)
                arr = np.frombuffer(buf, dtype=dtype).copy()
            else:
                arr = np.zeros(0, dtype=dtype)
            if name in ("h0", "h1", "h2"):
                arr = arr.reshape(-1, 2)
            out[name] = arr
        for name in SCALARS:
            out[name] = int(lib.oracle_scalar(h, name.encode()))
    finally:
        lib.oracle_free(h)
    return out


# ---- thresholds (threshold.py:20-200), in FP64 ---------------------------------------
def _sq_dists_f64(q, pts, qn, pn):
    """Squared distances of rows q to all pts in FP64 by the Gram expansion
    (relative error ~1e-15 of |x|^2, far below the fp32 values compared
    against it), clamped at 0."""
    return np.maximum(qn[:, None] + pn[None, :] - 2.0 * (q @ pts.T), 0.0)


def knn_kth_f64(points, k: int, chunk: int = 1024) -> np.ndarray:
    """k-th nearest-neighbour distance of every point (the point itself
    excluded, duplicates of it counted at distance 0), in FP64: the quantity
    ``_tiled_knn`` (threshold.py:133-176) computes with fp32 cdist tiles."""
    pts = np.asarray(points, dtype=np.float64)
    n = pts.shape[0]
    nrm = (pts * pts).sum(1)
    out = np.empty(n, dtype=np.float64)
    for s in range(0, n, chunk):
        q = pts[s:s + chunk]
        d2 = _sq_dists_f64(q, pts, nrm[s:s + chunk], nrm)
        d2[np.arange(q.shape[0]), np.arange(s, s + q.shape[0])] = np.inf
        out[s:s + chunk] = np.sqrt(np.partition(d2, k - 1, axis=1)[:, k - 1])
    return out


def auto_threshold_f64(points, k: int = 20, percentile: float = 95.0) -> float:
    """auto_threshold (threshold.py:20-78) without subsampling, in FP64: k
    clamped to [1, n - 1], percentile to [0, 100], linear-interpolation
    percentile of the k-th NN distances."""
    pts = np.asarray(points, dtype=np.float64)
    n = pts.shape[0]
    if n <= 1:
        return 0.0
    k = max(1, min(k, n - 1))
    percentile = max(0.0, min(100.0, percentile))
    return float(np.quantile(knn_kth_f64(pts, k), percentile / 100.0, method="linear"))


def enclosing_radius_f64(points, chunk: int = 1024) -> float:
    """enclosing_radius (threshold.py:81-116, 179-200) without subsampling,
    in FP64: min over points of the max distance to any point."""
    pts = np.asarray(points, dtype=np.float64)
    n = pts.shape[0]
    if n <= 1:
        return 0.0
    nrm = (pts * pts).sum(1)
    best = np.inf
    for s in range(0, n, chunk):
        d2 = _sq_dists_f64(pts[s:s + chunk], pts, nrm[s:s + chunk], nrm)
        best = min(best, float(np.sqrt(d2.max(axis=1)).min()))
    return best
