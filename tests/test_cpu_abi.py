"""CPU-only checks of the C ABI's host logic: argument checks that return a
status before any device work, their messages, and the pure size helpers.
No call here reaches the CUDA runtime."""
from __future__ import annotations

import ctypes

import pytest

from flashph_b200 import _build

PH_OK, PH_ERR_ARG, PH_ERR_CAPACITY, PH_ERR_OVERFLOW = 0, 2, 3, 6
NULL = None


@pytest.fixture(scope="module")
def lib():
    lib = ctypes.CDLL(_build.build())
    i64, i32, p = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p
    lib.ph_last_error.restype = ctypes.c_char_p
    lib.ph_cloud_tiles.restype = i64
    lib.ph_cloud_tiles.argtypes = [i64]
    lib.ph_edges_sort_noalloc_max_edges.restype = i64
    lib.ph_edges_sort_workspace_bytes.restype = ctypes.c_size_t
    lib.ph_edges_sort_workspace_bytes.argtypes = [i64]
    lib.ph_edges_sort.argtypes = [p, p, p, i64, i64, p, p, p, p, ctypes.c_size_t, p]
    lib.ph_edges_sort_noalloc.argtypes = [p, p, p, i64, i64, p, p, p, p]
    lib.ph_vertex_csr.argtypes = [p, p, i64, i64, p, p, p, p, ctypes.c_size_t, p]
    lib.ph_boruvka_mst.argtypes = [p, p, i64, i64, p, p, p, p, p, ctypes.c_size_t, p]
    lib.ph_knn_kth.argtypes = [p, i64, i32, i32, p, p]
    lib.ph_quantile_f32.argtypes = [p, i64, ctypes.c_double, p, p, ctypes.c_size_t, p]
    lib.ph_enclosing_radius.argtypes = [p, i64, i32, p, p, ctypes.c_size_t, p]
    lib.ph_rips_persistence.argtypes = [p, i64, i32, ctypes.c_double, i32, i64, i64, i32,
                                        ctypes.POINTER(p), p]
    return lib


def test_cloud_tiles_counts_upper_triangle_tiles(lib):
    # 128 x 128 point tiles over i <= j
    for n, nt in [(0, 0), (1, 0), (2, 1), (128, 1), (129, 2), (20000, 157)]:
        assert lib.ph_cloud_tiles(n) == (nt * (nt + 1) // 2 if n >= 2 else 0), n


def test_sort_sizes_are_checked_before_any_device_work(lib):
    assert lib.ph_edges_sort(NULL, NULL, NULL, -1, 10, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW
    assert lib.ph_edges_sort(NULL, NULL, NULL, 1 << 31, 10, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW
    assert lib.ph_edges_sort(NULL, NULL, NULL, 0, 10, NULL, NULL, NULL, NULL, 0, NULL) == PH_OK
    assert lib.ph_vertex_csr(NULL, NULL, -1, 10, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW
    assert lib.ph_vertex_csr(NULL, NULL, 5, -1, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW
    assert lib.ph_boruvka_mst(NULL, NULL, 5, -1, NULL, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW
    assert lib.ph_boruvka_mst(NULL, NULL, 1 << 31, 5, NULL, NULL, NULL, NULL, NULL, 0, NULL) == PH_ERR_OVERFLOW


def test_noalloc_sort_rejects_sizes_beyond_its_static_scratch(lib):
    cap = lib.ph_edges_sort_noalloc_max_edges()
    assert cap == 1 << 19
    assert lib.ph_edges_sort_noalloc(NULL, NULL, NULL, -1, 10, NULL, NULL, NULL, NULL) == PH_ERR_ARG
    assert lib.ph_edges_sort_noalloc(NULL, NULL, NULL, cap + 1, 10, NULL, NULL, NULL, NULL) == PH_ERR_CAPACITY
    assert b"524288" in lib.ph_last_error()
    # the static scratch holds the allocating sort's workspace for the largest allowed size
    assert lib.ph_edges_sort_workspace_bytes(cap) <= 13 << 20


def test_threshold_arguments(lib):
    assert lib.ph_knn_kth(NULL, -1, 3, 5, NULL, NULL) == PH_ERR_ARG
    assert lib.ph_knn_kth(NULL, 10, 0, 5, NULL, NULL) == PH_ERR_ARG
    assert lib.ph_knn_kth(NULL, 10, 3, 0, NULL, NULL) == PH_ERR_ARG
    assert lib.ph_knn_kth(NULL, 10, 3, 10, NULL, NULL) == PH_ERR_ARG  # k above n - 1
    assert lib.ph_knn_kth(NULL, 0, 3, 5, NULL, NULL) == PH_OK
    assert lib.ph_quantile_f32(NULL, 0, 0.5, NULL, NULL, 0, NULL) == PH_ERR_ARG
    assert lib.ph_quantile_f32(NULL, 10, 1.5, NULL, NULL, 0, NULL) == PH_ERR_ARG
    assert lib.ph_quantile_f32(NULL, 10, float("nan"), NULL, NULL, 0, NULL) == PH_ERR_ARG
    assert lib.ph_enclosing_radius(NULL, 0, 3, NULL, NULL, 0, NULL) == PH_ERR_ARG
    assert lib.ph_enclosing_radius(NULL, 10, 0, NULL, NULL, 0, NULL) == PH_ERR_ARG


def test_native_call_arguments_and_messages(lib):
    out = ctypes.c_void_p(123)
    pts = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert lib.ph_rips_persistence(pts, 10, 3, 1.0, 1, 0, 0, 0, None, NULL) == PH_ERR_ARG
    for args in [(NULL, 10, 3, 1.0, 1), (pts, 1, 3, 1.0, 1), (pts, 10, 0, 1.0, 1), (pts, 10, 3, 1.0, 3),
                 (pts, 10, 3, 1.0, -1)]:
        assert lib.ph_rips_persistence(*args, 0, 0, 0, ctypes.byref(out), NULL) == PH_ERR_ARG, args
        assert out.value is None
        assert b"invalid argument" in lib.ph_last_error()
    # the tensor-core screen takes d <= 252
    assert lib.ph_rips_persistence(pts, 10, 253, 1.0, 1, 0, 0, 1, ctypes.byref(out), NULL) == PH_ERR_ARG
    assert lib.ph_rips_persistence(pts, 1 << 31, 3, 1.0, 1, 0, 0, 0, ctypes.byref(out), NULL) == PH_ERR_OVERFLOW
    assert b"int32" in lib.ph_last_error()
