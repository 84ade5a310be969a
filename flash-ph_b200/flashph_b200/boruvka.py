"""H0: minimum spanning forest on the GPU (reference: boruvka.py)."""
from __future__ import annotations

import torch
from torch import Tensor

from . import _lib as L


def gpu_boruvka_mst(edge_i: Tensor, edge_j: Tensor, edge_rank: Tensor | None, n: int):
    """Minimum spanning forest under the edge ranks (= positions).

    Mirrors ``boruvka.py:17 gpu_boruvka_mst``: returns the sorted indices of
    the forest edges (int64) and the component label of every vertex (its
    smallest vertex index). ``edge_rank`` must be ``arange(E)``, as in every
    call of the reference; it is accepted for signature compatibility.
    """
    mask, comp, _ = boruvka_mask(edge_i, edge_j, n)
    return mask.nonzero(as_tuple=True)[0], comp.long()


def boruvka_mask(edge_i: Tensor, edge_j: Tensor, n: int):
    """Forest as a per-edge uint8 mask, labels and the component count tensor."""
    dev = edge_i.device
    E = edge_i.shape[0]
    mask = torch.empty(E, dtype=torch.uint8, device=dev)
    comp = torch.empty(n, dtype=torch.int32, device=dev)
    ncomp = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    nb = L.query("ph_boruvka_workspace_bytes", n, E)
    ws = L.workspace(nb, dev)
    L.call("ph_boruvka_mst", L.ptr(edge_i), L.ptr(edge_j), E, n, L.ptr(mask), L.ptr(comp),
           ncomp.data_ptr(), status.data_ptr(), ws.data_ptr(), nb, L.stream_handle(dev))
    return mask, comp, (ncomp, status)


def h0_rows(edge_filt: Tensor, mst_mask: Tensor, n: int) -> Tensor:
    """(0, death) rows of the forest edges ascending, then (0, inf) rows."""
    dev = edge_filt.device
    E = edge_filt.shape[0]
    rows = torch.empty(n, 2, dtype=torch.float32, device=dev)
    nb = L.query("ph_h0_rows_workspace_bytes", E)
    ws = L.workspace(nb, dev)
    L.call("ph_h0_rows", L.ptr(edge_filt), L.ptr(mst_mask), E, n, rows.data_ptr(), ws.data_ptr(), nb,
           L.stream_handle(dev))
    return rows
