"""Failure paths on the GPU, made on purpose without a device fault.

The reducer bounds every column's loop; a test makes that bound tiny
(ph_set_reduce_limits) so the loop gives up: the call reports
PH_ERR_ITER_LIMIT as a PHError and the context stays usable (the next call,
with the default bound, gives the oracle's diagrams). A first reduction pool
capped far below the need makes the pool run out: the native call retries
with a pool four times larger until the reduction fits, and the diagrams are
unchanged. The batched call takes the same path.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture
def limits():
    from flashph_b200 import _lib
    lib = _lib.lib()
    yield lib.ph_set_reduce_limits
    lib.ph_set_reduce_limits(0, 0)


def _cloud():
    return np.random.default_rng(3).standard_normal((600, 10)).astype(np.float32), 2.5


def test_iteration_limit_is_reported_and_the_context_survives(limits):
    from flashph_b200 import _lib, rips_persistence
    pts, t = _cloud()
    ref = oracle.run(pts, t, 1, fused=True)
    assert ref["xor_ops"] > 0  # some column needs more than one step
    limits(1, 0)
    with pytest.raises(_lib.PHError, match="iteration limit"):
        rips_persistence(torch.from_numpy(pts).cuda(), t, max_dim=1)
    limits(0, 0)
    got = rips_persistence(torch.from_numpy(pts).cuda(), t, max_dim=1)
    assert np.array_equal(_bits(got[1].cpu().numpy()), _bits(ref["h1"]))


def test_pool_exhaustion_is_retried_with_a_larger_pool(limits):
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import rips_persistence_batch
    pts, t = _cloud()
    want = rips_persistence(torch.from_numpy(pts).cuda(), t, max_dim=2)
    limits(0, 16384)  # below the initial records alone (33K H1, 66K H2 entries): the first attempt runs out
    got = rips_persistence(torch.from_numpy(pts).cuda(), t, max_dim=2)
    batched = rips_persistence_batch([pts, pts[:300]], [t, t], 2)
    limits(0, 0)
    for a, b in zip(want, got):
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b.cpu().numpy()))
    for a, b in zip(want, batched[0]):
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b.cpu().numpy()))


def test_pool_exhaustion_reported_by_the_reduction_entry_point():
    """ph_reduce itself with a pool too small: status PH_ERR_POOL."""
    from flashph_b200 import rips_persistence  # noqa: F401  (loads the library)
    from flashph_b200.cohomology import cof_max_face, cofacet_csr, emit_triangles, count_triangles, reduce
    from flashph_b200.boruvka import boruvka_mask
    from flashph_b200.rips import rips_filtration
    pts, t = _cloud()
    f = rips_filtration(torch.from_numpy(pts).cuda(), t)
    E = f.edge_i.shape[0]
    mst, _, _ = boruvka_mask(f.edge_i, f.edge_j, pts.shape[0])
    tri_off = count_triangles(f)
    T = int(tri_off[-1].item())
    tris = emit_triangles(f, tri_off, T)
    off, data = cofacet_csr(E, E, T, 3, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb)
    cmf = cof_max_face(T, 3, 0, mst, f0=tris.tri_m, f1=tris.tri_fa, f2=tris.tri_fb)
    red = reduce(off, data, E, 0, T, E, mst, cmf, 64)
    assert int(red.status.item()) == 5  # PH_ERR_POOL
