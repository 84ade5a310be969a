"""The no-allocation filtration sort, through the C ABI.

``ph_edges_sort_noalloc`` serves callers that cannot allocate device memory
(their HBM belongs to another allocator or a fixed budget): it takes only
inputs and outputs and keeps its scratch in a static device array. Its
output must equal the allocating ``ph_edges_sort`` bit for bit (the sort is
integer work), on consecutive calls that share that array. This file is
collected last so that a run stopping at the first failure has run every
other test before it.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _edges(E, n, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(n * (n - 1) // 2, size=E, replace=False)
    j = np.floor((1 + np.sqrt(1 + 8 * flat.astype(np.float64))) / 2).astype(np.int64)
    j = np.where(j * (j - 1) // 2 > flat, j - 1, j)
    j = np.where((j + 1) * j // 2 <= flat, j + 1, j)
    i = flat - j * (j - 1) // 2
    dsq = rng.integers(0, 40, size=E).astype(np.float32) / np.float32(3.0)
    return (torch.from_numpy(i.astype(np.int32)).cuda(), torch.from_numpy(j.astype(np.int32)).cuda(),
            torch.from_numpy(dsq).cuda())


def _allocating_sort(lib, ei, ej, ed, n, stream):
    E = ei.numel()
    out = [torch.empty_like(ei), torch.empty_like(ej), torch.empty_like(ed)]
    nb = lib.ph_edges_sort_workspace_bytes(E)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device="cuda")
    rc = lib.ph_edges_sort(ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), E, n, out[0].data_ptr(),
                           out[1].data_ptr(), out[2].data_ptr(), ws.data_ptr(), nb, stream)
    assert rc == 0
    return out


def _noalloc_sort(lib, ei, ej, ed, n, stream):
    E = ei.numel()
    out = [torch.empty_like(ei), torch.empty_like(ej), torch.empty_like(ed)]
    rc = lib.ph_edges_sort_noalloc(ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), E, n, out[0].data_ptr(),
                                   out[1].data_ptr(), out[2].data_ptr(), stream)
    assert rc == 0, lib.ph_last_error()
    return out


def test_noalloc_sort_matches_allocating_sort_on_consecutive_calls():
    from flashph_b200 import _lib
    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cap = lib.ph_edges_sort_noalloc_max_edges()
    assert cap == 1 << 19
    # Two calls in a row that both keep their scratch in the static array (the
    # multi-launch radix form: more than 98,304 edges, n > 92682, which also
    # takes the colex-collision path): the second, smaller call starts on the
    # first call's leftover control block and look-back flags. A third call
    # below the cluster form's limit (no scratch at all) closes the sequence.
    for E, n, seed in ((cap, 200000, 2), (150000, 120000, 3), (70000, 5000, 1)):
        ei, ej, ed = _edges(E, n, seed)
        want = _allocating_sort(lib, ei, ej, ed, n, stream)
        got = _noalloc_sort(lib, ei, ej, ed, n, stream)
        torch.cuda.synchronize()
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])
        assert torch.equal(got[2].view(torch.int32), want[2].view(torch.int32))
        # the order is the packed-key order
        key = (want[2].view(torch.int32).long() << 32) | (
            (want[1].long() * (want[1].long() - 1) // 2 + want[0].long()) & 0xFFFFFFFF)
        assert bool((key[1:] >= key[:-1]).all())


def test_noalloc_sort_rejects_more_edges_than_its_scratch_holds():
    from flashph_b200 import _lib
    lib = _lib.lib()
    cap = lib.ph_edges_sort_noalloc_max_edges()
    E = cap + 1
    rc = lib.ph_edges_sort_noalloc(None, None, None, E, 10 ** 6, None, None, None,
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == 3  # PH_ERR_CAPACITY, raised before any device work
    assert b"524288" in lib.ph_last_error()
