"""Threshold estimation (reference: threshold.py).

``auto_threshold``: percentile of k-th nearest-neighbour distances;
``enclosing_radius``: min over points of the max distance to any point.
Same signatures, defaults, clamping and subsampling as the reference; the
distance scans, the sort and the quantile run in the CUDA library.
"""
from __future__ import annotations

import numpy as np
import torch
from torch import Tensor

from . import _lib as L


def _to_tensor(points) -> Tensor:
    if isinstance(points, np.ndarray):
        t = torch.from_numpy(points).float()
        if torch.cuda.is_available():
            t = t.cuda()
        return t
    return points.float()


def _on_cuda(pts: Tensor) -> Tensor:
    if pts.device.type != "cuda":
        if not torch.cuda.is_available():
            raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
        pts = pts.cuda()
    return pts.contiguous()


def knn_kth_distance(pts: Tensor, k: int) -> Tensor:
    """(n,) k-th nearest-neighbour distance of every point (self excluded)."""
    pts = _on_cuda(pts)
    n, d = pts.shape
    out = torch.empty(n, dtype=torch.float32, device=pts.device)
    L.call("ph_knn_kth", pts.data_ptr(), n, d, k, out.data_ptr(), L.stream_handle(pts.device))
    return out


def quantile(values: Tensor, q: float) -> Tensor:
    """torch.quantile(values, q) (linear interpolation) on the GPU; 0-d tensor."""
    n = values.numel()
    out = torch.empty(1, dtype=torch.float32, device=values.device)
    nb = L.query("ph_quantile_workspace_bytes", n)
    ws = L.workspace(nb, values.device)
    L.call("ph_quantile_f32", values.contiguous().data_ptr(), n, float(q), out.data_ptr(), ws.data_ptr(), nb,
           L.stream_handle(values.device))
    return out[0]


def auto_threshold(points, k: int = 20, percentile: float = 95.0, subsample: int | None = None) -> float:
    """Estimate a Rips threshold from the k-NN distance distribution.

    Mirrors ``threshold.py:20-78``: k is clamped to [1, n-1], an optional
    random subsample is drawn first, the percentile is clamped to [0, 100]
    and the linear-interpolation percentile of the k-th NN distances is
    returned as a Python float.
    """
    pts = _to_tensor(points)
    n = pts.shape[0]
    if n <= 1:
        return 0.0
    k = max(1, min(k, n - 1))
    if subsample is not None and subsample >= 2 and subsample < n:
        idx = torch.randperm(n, device=pts.device)[:subsample]
        pts = pts[idx]
        n = pts.shape[0]
        k = max(1, min(k, n - 1))
    percentile = max(0.0, min(100.0, percentile))
    knn = knn_kth_distance(pts, k)
    return float(quantile(knn, percentile / 100.0).item())


def enclosing_radius(points, subsample: int | None = None) -> float:
    """min over x of max over y of d(x, y) (threshold.py:81-116)."""
    pts = _to_tensor(points)
    n = pts.shape[0]
    if n <= 1:
        return 0.0
    if subsample is not None and subsample >= 2 and subsample < n:
        idx = torch.randperm(n, device=pts.device)[:subsample]
        pts = pts[idx]
    pts = _on_cuda(pts)
    n, d = pts.shape
    out = torch.empty(1, dtype=torch.float32, device=pts.device)
    nb = L.query("ph_enclosing_radius_workspace_bytes", n)
    ws = L.workspace(nb, pts.device)
    L.call("ph_enclosing_radius", pts.data_ptr(), n, d, out.data_ptr(), ws.data_ptr(), nb,
           L.stream_handle(pts.device))
    return float(out.item())
