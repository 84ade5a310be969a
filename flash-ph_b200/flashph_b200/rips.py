"""Vietoris-Rips filtration on the B200 (reference: rips.py).

``rips_filtration`` returns the same ``RipsFiltration`` record as the
reference (``rips.py:15-27``): edges sorted by the packed key
(dist^2 bits, 32-bit colex), and the per-vertex adjacency with edge ranks.
All arithmetic runs in the CUDA library; this module only allocates and
sequences.
"""
from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from . import _timing

# Initial edge-buffer capacity; a run with more edges is repeated once with
# the exact count.
_MIN_EDGE_CAPACITY = 1 << 22
# ph_cloud_seg (include/flashph_b200.h)
_SEG_DTYPE = np.dtype([("pt_off", "<i8"), ("vbase", "<i8"), ("tile_off", "<i8"), ("n", "<i4"), ("d", "<i4"),
                       ("thr_sq", "<f4"), ("max_dim", "<i4")])


class RipsFiltration(NamedTuple):
    """Result of Rips filtration construction (edges in filtration order)."""
    edge_i: Tensor        # (E,) int32, i < j
    edge_j: Tensor        # (E,) int32
    edge_dist_sq: Tensor  # (E,) float32
    vert_adj_ptr: Tensor  # (n+1,) int32
    vert_adj_idx: Tensor  # (2E,) int32
    vert_adj_rank: Tensor  # (2E,) int32
    vert_adj_dist_sq: Tensor  # (2E,) float32 (kept for the record layout; filled on request)
    n: int


def threshold_sq(max_edge_length: float) -> float:
    """fp32 of the double product t*t, as the reference's kernel argument
    (inf when the product exceeds the fp32 range)."""
    with np.errstate(over="ignore"):
        return float(np.float32(float(max_edge_length) * float(max_edge_length)))


def enumerate_edges(points: Tensor, max_edge_length: float, screen: bool | None = None, stats: bool = False):
    """Unsorted edges (i, j, dist^2) of all pairs with dist^2 < fp32(t*t).

    ``screen`` forces the tensor-core screened kernel (True) or the direct
    kernel (False); None picks by dimension. Both give the same edges."""
    from ._edges import enumerate_segments

    dev = points.device
    n, d = points.shape
    seg = np.zeros(1, dtype=_SEG_DTYPE)
    seg[0] = (0, 0, 0, n, d, threshold_sq(max_edge_length), 1)
    seg_dev = torch.from_numpy(seg.view(np.uint8).copy()).to(dev, non_blocking=True)
    pairs = n * (n - 1) // 2
    cap = int(min(pairs, max(_MIN_EDGE_CAPACITY, 256 * n)))
    return enumerate_segments(points, seg, seg_dev, int(L.query("ph_cloud_tiles", n)), cap, screen, stats)


def sort_edges(ei: Tensor, ej: Tensor, ed: Tensor, n: int):
    dev = ei.device
    E = ei.shape[0]
    oi = torch.empty_like(ei)
    oj = torch.empty_like(ej)
    od = torch.empty_like(ed)
    if E:
        nb = L.query("ph_edges_sort_workspace_bytes", E)
        ws = L.workspace(nb, dev)
        L.call("ph_edges_sort", ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), E, n, oi.data_ptr(),
               oj.data_ptr(), od.data_ptr(), ws.data_ptr(), nb, L.stream_handle(dev))
    return oi, oj, od


def vertex_csr(ei: Tensor, ej: Tensor, n: int):
    dev = ei.device
    E = ei.shape[0]
    ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    idx = torch.empty(2 * E, dtype=torch.int32, device=dev)
    rank = torch.empty(2 * E, dtype=torch.int32, device=dev)
    nb = L.query("ph_vertex_csr_workspace_bytes", E)
    ws = L.workspace(nb, dev)
    L.call("ph_vertex_csr", L.ptr(ei), L.ptr(ej), E, n, ptr.data_ptr(), L.ptr(idx), L.ptr(rank),
           ws.data_ptr(), nb, L.stream_handle(dev))
    return ptr, idx, rank


def rips_filtration(points: Tensor, max_edge_length: float) -> RipsFiltration:
    """Construct the Rips filtration of an (n, d) CUDA point cloud."""
    if max_edge_length < 0:
        raise ValueError(f"max_edge_length must be non-negative, got {max_edge_length}")
    n, d = points.shape
    dev = points.device
    if dev.type != "cuda":
        raise RuntimeError("rips_filtration needs a CUDA tensor")
    pts = points.float().contiguous()
    e32 = torch.empty(0, dtype=torch.int32, device=dev)
    f32 = torch.empty(0, dtype=torch.float32, device=dev)
    if n <= 1:
        return RipsFiltration(e32, e32, f32, torch.zeros(n + 1, dtype=torch.int32, device=dev),
                              e32, e32, f32, n)
    ei, ej, ed = enumerate_edges(pts, max_edge_length)
    with _timing.stage("sort"):
        ei, ej, ed = sort_edges(ei, ej, ed, n)
    with _timing.stage("vertex_csr"):
        ptr, idx, rank = vertex_csr(ei, ej, n)
    return RipsFiltration(ei, ej, ed, ptr, idx, rank, f32, n)


def edge_filtration_values(edge_dist_sq: Tensor) -> Tensor:
    """sqrt of dist^2, correctly rounded (reduce_h1_gpu.py:479)."""
    out = torch.empty_like(edge_dist_sq)
    if edge_dist_sq.numel():
        L.call("ph_sqrt_f32", edge_dist_sq.data_ptr(), out.data_ptr(), edge_dist_sq.numel(),
               L.stream_handle(edge_dist_sq.device))
    return out
