"""ctypes binding of the C ABI in ``include/flashph_b200.h``.

The shared library is the only compute path: if it cannot be loaded, every
entry point raises. Device memory, streams and counts come from torch;
pointers go to the library as plain integers.
"""
from __future__ import annotations

import ctypes
import os

import torch

from . import _build

_LIB = None

PH_OK = 0
_STATUS = {1: "CUDA error", 2: "invalid argument", 3: "capacity exceeded",
           4: "iteration limit reached", 5: "reduction pool exhausted", 6: "count overflow",
           7: "limit exceeded"}

P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int32
F32 = ctypes.c_float
F64 = ctypes.c_double
SZ = ctypes.c_size_t

# name -> (restype, argtypes)
_SIGS = {
    "ph_version": (ctypes.c_int, []),
    "ph_last_error": (ctypes.c_char_p, []),
    "ph_launch_count": (ctypes.c_ulonglong, []),
    "ph_edges_enumerate": (ctypes.c_int, [P, I64, I32, F32, P, P, P, I64, P, P]),
    "ph_edges_sort_workspace_bytes": (SZ, [I64]),
    "ph_edges_sort": (ctypes.c_int, [P, P, P, I64, I64, P, P, P, P, SZ, P]),
    "ph_edges_sort_noalloc_max_edges": (I64, []),
    "ph_edges_sort_noalloc": (ctypes.c_int, [P, P, P, I64, I64, P, P, P, P]),
    "ph_vertex_csr_workspace_bytes": (SZ, [I64]),
    "ph_vertex_csr": (ctypes.c_int, [P, P, I64, I64, P, P, P, P, SZ, P]),
    "ph_sqrt_f32": (ctypes.c_int, [P, P, I64, P]),
    "ph_boruvka_workspace_bytes": (SZ, [I64, I64]),
    "ph_boruvka_mst": (ctypes.c_int, [P, P, I64, I64, P, P, P, P, P, SZ, P]),
    "ph_h0_rows_workspace_bytes": (SZ, [I64]),
    "ph_h0_rows": (ctypes.c_int, [P, P, I64, I64, P, P, SZ, P]),
    "ph_triangles_count_workspace_bytes": (SZ, [I64]),
    "ph_triangles_count": (ctypes.c_int, [P, P, I64, P, P, P, P, P, P, SZ, P]),
    "ph_triangles_emit": (ctypes.c_int, [P, P, I64, P, P, P, P, P, P, P, P, P]),
    "ph_tets_count_workspace_bytes": (SZ, [I64]),
    "ph_tets_count": (ctypes.c_int, [P, P, I64, P, P, P, P, P, P, SZ, P]),
    "ph_tets_emit": (ctypes.c_int, [P, P, I64, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "ph_cloud_tiles": (I64, [I64]),
    "ph_rips_persistence": (ctypes.c_int, [P, I64, I32, ctypes.c_double, I32, I64, I64, I32,
                                           ctypes.POINTER(ctypes.c_void_p), P]),
    "ph_result_rows": (I64, [P, I32]),
    "ph_result_stat": (I64, [P, I32]),
    "ph_result_copy": (ctypes.c_int, [P, I32, P, I32, P]),
    "ph_result_copy_all": (ctypes.c_int, [P, P, I32, P]),
    "ph_set_dependent_launch": (None, [I32]),
    "ph_set_reduce_limits": (None, [I64, I64]),
    "ph_probe_l2_chase": (ctypes.c_int, [P, I32, ctypes.c_uint32, P, P]),
    "ph_triangles_total_edges_workspace_bytes": (SZ, [I64, I64]),
    "ph_triangles_total_edges": (ctypes.c_int, [P, P, I64, I64, P, P, SZ, P]),
    "ph_result_free": (None, [P]),
    "ph_rips_persistence_batch": (ctypes.c_int, [P, P, P, P, P, I32, I64, I64, I32, I64,
                                                 ctypes.POINTER(ctypes.c_void_p), P]),
    "ph_batch_result_status": (I32, [P, I32]),
    "ph_batch_result_message": (ctypes.c_char_p, [P, I32]),
    "ph_batch_result_stat": (I64, [P, I32, I32]),
    "ph_batch_result_offsets": (ctypes.c_int, [P, I32, P]),
    "ph_batch_result_copy": (ctypes.c_int, [P, I32, P, I32, P]),
    "ph_batch_result_free": (None, [P]),
    "ph_triangles_total_max_vertices": (I64, []),
    "ph_triangles_total": (ctypes.c_int, [P, P, I64, P, P, P]),
    "ph_batch_triangles_total": (ctypes.c_int, [P, P, I64, P, P, I32, P, P, P]),
    "ph_edges_screened_workspace_bytes": (SZ, [I64, I32, I32]),
    "ph_batch_edges_enumerate_screened": (ctypes.c_int, [P, P, I32, I64, I32, I64, P, I64, P, P, P, I64, P, P, P,
                                                         P, SZ, P]),
    "ph_batch_edges_enumerate": (ctypes.c_int, [P, P, I32, I64, P, P, P, I64, P, P]),
    "ph_batch_vertex_cloud": (ctypes.c_int, [P, I32, P, P]),
    "ph_batch_edges_sort_workspace_bytes": (SZ, [I64]),
    "ph_batch_edges_sort": (ctypes.c_int, [P, P, P, I64, P, P, I32, I32, P, P, P, P, SZ, P]),
    "ph_batch_item_offsets": (ctypes.c_int, [P, I64, P, I32, P, P]),
    "ph_batch_h0_rows_workspace_bytes": (SZ, [I64]),
    "ph_batch_h0_rows": (ctypes.c_int, [P, P, I64, P, P, I32, P, I64, P, P, SZ, P]),
    "ph_batch_persistence_rows_workspace_bytes": (SZ, [I64]),
    "ph_batch_persistence_rows": (ctypes.c_int, [P, P, I64, I32, P, P, P, P, I32, P, P, P, P, SZ, P]),
    "ph_batch_edge_dim_mask": (ctypes.c_int, [P, I64, P, P, I32, P, P]),
    "ph_or_gather_mask": (ctypes.c_int, [P, P, P, I64, I32, P]),
    "ph_batch_knn_kth": (ctypes.c_int, [P, P, I32, P, I64, I32, I32, P, P]),
    "ph_batch_quantile_workspace_bytes": (SZ, [I64]),
    "ph_batch_quantile": (ctypes.c_int, [P, I64, P, P, I32, F64, P, P, SZ, P]),
    "ph_cofacet_csr_workspace_bytes": (SZ, [I64, I32]),
    "ph_cofacet_csr": (ctypes.c_int, [P, P, P, P, I32, I64, I64, I32, P, P, P, SZ, P]),
    "ph_cof_max_face": (ctypes.c_int, [P, P, P, P, I32, I64, I32, P, P, P]),
    "ph_cofacet_rows3_max_row": (I32, []),
    "ph_cofacet_rows3_workspace_bytes": (SZ, [I64]),
    "ph_cofacet_rows3": (ctypes.c_int, [P, P, P, I64, I64, I32, P, I32, P, P, P, P, SZ, P]),
    "ph_max_count": (ctypes.c_int, [P, I64, P, P]),
    "ph_reduce_workspace_bytes": (SZ, [I64, I64, I64]),
    "ph_reduce": (ctypes.c_int, [P, P, I64, I32, I64, I32, I64, P, P, P, P, P, I64, P, P, P, SZ, P]),
    "ph_mark_pivots": (ctypes.c_int, [P, P, I64, I32, P, I64, P]),
    "ph_persistence_rows_workspace_bytes": (SZ, [I64]),
    "ph_persistence_rows": (ctypes.c_int, [P, P, I64, I32, P, P, P, P, P, P, SZ, P]),
    "ph_knn_kth": (ctypes.c_int, [P, I64, I32, I32, P, P]),
    "ph_quantile_workspace_bytes": (SZ, [I64]),
    "ph_quantile_f32": (ctypes.c_int, [P, I64, F64, P, P, SZ, P]),
    "ph_enclosing_radius_workspace_bytes": (SZ, [I64]),
    "ph_enclosing_radius": (ctypes.c_int, [P, I64, I32, P, P, SZ, P]),
}


class PHError(RuntimeError):
    """A library entry point returned a failure status."""

    def __init__(self, name: str, code: int, detail: str = ""):
        self.code = code
        msg = f"{name} failed: {_STATUS.get(code, code)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


def lib():
    """The loaded CUDA library (built on first use if missing)."""
    global _LIB
    if _LIB is None:
        # the library must be the build of the sources next to it (the entry
        # points' argument lists above follow those sources): rebuilt when
        # missing or when the sources' digest differs from its build stamp
        path = _build.build()
        handle = ctypes.CDLL(path)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def library_path() -> str:
    return _build.LIB_PATH


def call(name: str, *args) -> None:
    """Call a status-returning entry point; raise PHError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != PH_OK:
        detail = lib().ph_last_error().decode(errors="replace") if rc == 1 else ""
        raise PHError(name, rc, detail)


def query(name: str, *args) -> int:
    return int(getattr(lib(), name)(*args))


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if t.numel() == 0:
        return None
    return t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def check_status(name: str, status: torch.Tensor) -> None:
    """Raise if a device status word is non-zero (synchronises)."""
    st = int(status.item())
    if st != PH_OK:
        raise PHError(name, st)


def launch_count() -> int:
    """Kernels launched by the CUDA library in this process so far."""
    return int(lib().ph_launch_count())
