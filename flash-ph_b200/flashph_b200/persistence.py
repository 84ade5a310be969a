"""Public API: Vietoris-Rips persistent homology (H0, H1, H2) on the B200.

Mirrors ``persistence.py:77-215`` of the reference: the same signature,
validation messages, edge cases and output convention (a list of
``max_dim + 1`` float32 ``(K, 2)`` tensors on the input's device, ``inf``
deaths for essential classes). Every stage runs in the CUDA library; there is
no CPU path. CPU tensors and numpy arrays are moved to the current CUDA
device and the results are returned on the input's device.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch
from torch import Tensor

from . import _lib as L
from . import _timing
from ._lib import check_status
from .boruvka import boruvka_mask, h0_rows
from .cohomology import h1_diagram, h2_diagram
from .rips import edge_filtration_values, rips_filtration

_VERTEX_PACK_BITS = 16
_VALID_BACKENDS = ("auto", "gpu", "giotto")


def _empty(device, k=0):
    return torch.empty(k, 2, dtype=torch.float32, device=device)


def rips_persistence(
    points,
    max_edge_length: float,
    max_dim: int = 1,
    backend: str = "auto",
) -> list[Tensor]:
    """Exact Vietoris-Rips persistent homology (H0 + H1 + optional H2).

    Parameters
    ----------
    points : (n, d) array-like
        Point cloud (numpy arrays are moved to CUDA, as in the reference).
    max_edge_length : float
        Edges are kept when dist^2 < fp32(max_edge_length^2) (strict).
    max_dim : int
        0, 1 or 2. H2 requires n < 65536.
    backend : str
        Accepted for compatibility ('auto', 'gpu', 'giotto'); every value
        runs the CUDA reduction.

    Returns
    -------
    list[Tensor]
        [H0, H1, ...], each (K, 2) float32 on the input's device.
    """
    if isinstance(points, np.ndarray):
        points = torch.from_numpy(points).float()
        if torch.cuda.is_available():
            points = points.cuda()
    if max_edge_length < 0:
        raise ValueError(f"max_edge_length must be non-negative, got {max_edge_length}")
    if points.ndim != 2:
        raise ValueError(f"points must have shape (n, d), got {tuple(points.shape)}")
    if max_dim not in (0, 1, 2):
        raise ValueError(f"max_dim must be 0, 1, or 2, got {max_dim}")
    if max_dim == 2 and points.shape[0] >= (1 << _VERTEX_PACK_BITS):
        raise ValueError(
            f"H2 requires n < {1 << _VERTEX_PACK_BITS} (16-bit vertex packing), "
            f"got n={points.shape[0]}. Use max_dim=1 or reduce n.")
    if max_dim == 1 and backend not in _VALID_BACKENDS:
        raise ValueError(f"backend must be one of {_VALID_BACKENDS}, got {backend!r}")

    out_device = points.device
    n = points.shape[0]
    if n == 0:
        return [_empty(out_device) for _ in range(max_dim + 1)]
    if n == 1:
        h0 = torch.tensor([[0.0, float("inf")]], dtype=torch.float32, device=out_device)
        return [h0] + [_empty(out_device) for _ in range(max_dim)]

    if points.device.type != "cuda":
        if not torch.cuda.is_available():
            raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
        points = points.cuda(non_blocking=points.is_pinned())
    dev = points.device
    with torch.cuda.device(dev):
        if os.environ.get("FLASHPH_PIPELINE", "native") == "staged":
            dgms = _compute_staged(points, float(max_edge_length), max_dim)
        else:
            return _compute_native(points.float().contiguous(), float(max_edge_length), max_dim, out_device)
    if out_device != dev:
        dgms = [d.to(out_device) for d in dgms]
    return dgms


_EDGE_MODES = {"auto": 0, "on": 1, "off": 2}


def _compute_native(points: Tensor, t: float, max_dim: int, out_device, max_triangles: int = 10_000_000,
                    max_tetrahedra: int = 10_000_000) -> list[Tensor]:
    """The whole call in the CUDA library (ph_rips_persistence); diagrams are
    copied straight to the caller's device (pinned host memory for CPU
    callers)."""
    n, d = points.shape
    dev = points.device
    mode = _EDGE_MODES.get(os.environ.get("FLASHPH_EDGE_SCREEN", "auto").lower(), 0)
    if mode == 1 and d > 252:
        mode = 2
    s = L.stream_handle(dev)
    res = ctypes.c_void_p()
    lib = L.lib()
    with _timing.stage("native"):
        rc = lib.ph_rips_persistence(points.data_ptr(), n, d, t, max_dim, max_triangles, max_tetrahedra, mode,
                                     ctypes.byref(res), s)
    if rc != L.PH_OK:
        msg = lib.ph_last_error().decode(errors="replace")
        if rc == 7:  # PH_ERR_LIMIT: the reference raises ValueError with this text
            raise ValueError(msg)
        raise L.PHError("ph_rips_persistence", rc, msg)
    try:
        to_host = out_device.type != "cuda"
        rows = [int(lib.ph_result_rows(res, k)) for k in range(max_dim + 1)]
        # one buffer and one copy call for all diagrams; the diagrams are views of it
        if to_host:
            buf = torch.empty(sum(rows), 2, dtype=torch.float32, pin_memory=True)
        else:
            buf = torch.empty(sum(rows), 2, dtype=torch.float32, device=out_device)
        L.call("ph_result_copy_all", res, buf.data_ptr(), 1 if to_host else 0, s)
        outs = list(buf.split(rows))
    finally:
        lib.ph_result_free(res)
    if to_host:
        torch.cuda.current_stream(dev).synchronize()
    return outs


def _compute_staged(points: Tensor, t: float, max_dim: int) -> list[Tensor]:
    """The same computation stage by stage from Python (each stage its own
    library call); kept as a cross-check of the native pipeline and for the
    stage-level timers."""
    n = points.shape[0]
    with _timing.stage("filtration"):
        filt = rips_filtration(points, t)
    with _timing.stage("h0"):
        edge_filt = edge_filtration_values(filt.edge_dist_sq)
        mst_mask, _, (_, mst_status) = boruvka_mask(filt.edge_i, filt.edge_j, n)
        h0 = h0_rows(edge_filt, mst_mask, n)
    if max_dim == 0:
        check_status("ph_boruvka_mst", mst_status)
        return [h0]
    with _timing.stage("h1"):
        h1, tris, red1, _ = h1_diagram(filt, edge_filt, mst_mask, checks=[("ph_boruvka_mst", mst_status)])
    if max_dim == 1:
        return [h0, h1]
    with _timing.stage("h2"):
        h2, _, _, _ = h2_diagram(filt, edge_filt, tris, red1)
    return [h0, h1, h2]
