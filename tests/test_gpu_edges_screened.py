"""Precision form: the tensor-core screened edge kernel returns exactly the
edges (pairs and dist^2 bits) of the direct FP32 kernel, on clouds chosen to
stress the screen's certified margin: every dimension class, clouds far from
the origin, duplicates and lattice ties on the strict threshold, tiny and
huge scales, anisotropic clouds, non-finite coordinates and huge thresholds
(tiles recomputed without the screen), ragged batches of mixed dimension."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from golden_util import sorted_rows

pytestmark = pytest.mark.gpu


def _edges(pts, t, screen):
    from flashph_b200.rips import enumerate_edges
    x = torch.as_tensor(np.ascontiguousarray(pts, dtype=np.float32)).cuda()
    ei, ej, ed = enumerate_edges(x, t, screen=screen, stats=screen)
    i, j, dsq = ei.cpu().numpy(), ej.cpu().numpy(), ed.cpu().numpy().view(np.uint32)
    o = np.lexsort((j, i))
    return i[o], j[o], dsq[o]


def _check(pts, t, expect_screened=True):
    from flashph_b200 import _edges as E
    a = _edges(pts, t, False)
    b = _edges(pts, t, True)
    assert a[0].shape == b[0].shape, (a[0].shape, b[0].shape)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    st = dict(E.last_screen_stats)
    n = len(pts)
    pairs = n * (n - 1) // 2
    if expect_screened:
        assert st["forced"] == 0, st
        # the screen passes every edge; far fewer pairs than all of them on sparse cases
        assert st["candidates"] >= len(a[0])
    return len(a[0]), st, pairs


def _quantile_t(pts, q, sample=400, seed=0):
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(pts), size=min(sample, len(pts)), replace=False)
    s = pts[idx].astype(np.float64)
    d = np.sqrt(((s[:, None, :] - s[None, :, :]) ** 2).sum(-1))
    return float(np.quantile(d[np.triu_indices(len(s), 1)], q))


@pytest.mark.parametrize("d", [1, 2, 3, 7, 8, 10, 12, 16, 17, 28, 31, 32, 50, 60, 61, 64, 65, 100, 128, 200, 252])
def test_gaussian_every_dimension(d):
    rng = np.random.default_rng(1000 + d)
    n = 1500 + 37 * (d % 5)
    pts = rng.standard_normal((n, d)).astype(np.float32)
    for q in (0.002, 0.05):
        E, st, pairs = _check(pts, _quantile_t(pts, q))
        assert E > 0


def test_sparse_screen_is_selective():
    rng = np.random.default_rng(7)
    pts = rng.standard_normal((6000, 50)).astype(np.float32)
    E, st, pairs = _check(pts, _quantile_t(pts, 0.001))
    assert st["candidates"] < pairs // 20, (st, pairs)


def test_far_from_origin_and_offset_dims():
    rng = np.random.default_rng(8)
    pts = (rng.standard_normal((3000, 10)) + 1.0e4).astype(np.float32)
    _check(pts, _quantile_t(pts, 0.01))
    pts = rng.standard_normal((3000, 33)).astype(np.float32)
    pts[:, 5] += 3.0e5
    pts[:, 20] -= 7.0e3
    _check(pts, _quantile_t(pts, 0.02))


def test_duplicates_and_lattice_ties_on_the_strict_threshold():
    g = np.stack(np.meshgrid(*[np.arange(6)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)
    pts = np.concatenate([g, g, g[::3]])  # exact duplicates (distance 0)
    pts = np.concatenate([pts, np.zeros((len(pts), 7), np.float32)], axis=1)  # d = 10
    for t in (1.0, float(np.sqrt(np.float32(2.0))), 2.0, 1.5, 0.0):
        _check(pts, t)
    # scaled lattice: distances exactly at the threshold after fp32 rounding
    _check(pts * np.float32(0.1), 0.1)


def test_tiny_and_huge_scales():
    rng = np.random.default_rng(9)
    base = rng.standard_normal((2000, 12))
    for scale in (1e-18, 1e-8, 1e8, 1e15):
        pts = (base * scale).astype(np.float32)
        _check(pts, _quantile_t(pts, 0.02))


def test_anisotropic_cloud():
    rng = np.random.default_rng(10)
    pts = rng.standard_normal((4000, 40))
    pts[:, 0] *= 1000.0
    pts[:, 1:] *= 0.01
    pts = pts.astype(np.float32)
    _check(pts, _quantile_t(pts, 0.01))


def test_nonfinite_and_huge_points_use_exact_tiles():
    from flashph_b200 import _edges as E
    rng = np.random.default_rng(11)
    pts = rng.standard_normal((700, 16)).astype(np.float32)
    pts[5, 3] = np.nan
    pts[300, 0] = np.inf
    _check(pts, 2.5, expect_screened=False)
    assert E.last_screen_stats["forced"] > 0
    pts = rng.standard_normal((500, 10)).astype(np.float32) * np.float32(1e37)
    _check(pts, 3e37, expect_screened=False)
    assert E.last_screen_stats["forced"] > 0


def test_huge_threshold_and_small_n():
    rng = np.random.default_rng(12)
    pts = rng.standard_normal((300, 20)).astype(np.float32)
    E, st, pairs = _check(pts, 1e20, expect_screened=False)  # fp32(t*t) = inf: every pair
    assert E == pairs
    for n in (2, 3, 127, 128, 129, 255, 257):
        p = rng.standard_normal((n, 9)).astype(np.float32)
        _check(p, 3.0)
    p = rng.standard_normal((1, 9)).astype(np.float32)
    assert _edges(p, 3.0, True)[0].size == 0


def test_batch_mixed_dimensions_screened_equals_direct(monkeypatch):
    from flashph_b200.batch import rips_persistence_batch
    rng = np.random.default_rng(13)
    clouds, ts = [], []
    for k in range(40):
        n = int(np.exp(rng.uniform(np.log(20), np.log(900))))
        d = [3, 8, 32, 50][k % 4]
        p = rng.standard_normal((n, d)).astype(np.float32)
        if k % 5 == 0:
            p += 50.0
        clouds.append(p)
        ts.append(_quantile_t(p, 0.03, seed=k))
    out = {}
    for mode in ("off", "on"):
        monkeypatch.setenv("FLASHPH_EDGE_SCREEN", mode)
        out[mode] = rips_persistence_batch(clouds, ts, 1)
    for a, b in zip(out["off"], out["on"]):
        assert not isinstance(a, Exception) and not isinstance(b, Exception)
        for da, db in zip(a, b):
            assert np.array_equal(da.cpu().numpy().view(np.uint32), db.cpu().numpy().view(np.uint32))


def test_persistence_through_screen_matches_oracle(monkeypatch):
    import oracle
    from flashph_b200 import rips_persistence
    rng = np.random.default_rng(14)
    pts = rng.standard_normal((900, 32)).astype(np.float32)
    t = _quantile_t(pts, 0.02)
    monkeypatch.setenv("FLASHPH_EDGE_SCREEN", "on")
    got = rips_persistence(torch.from_numpy(pts).cuda(), t, max_dim=2)
    ref = oracle.run(pts, t, 2, fused=True)
    for dim, key in enumerate(("h0", "h1", "h2")):
        g = sorted_rows(got[dim].cpu().numpy())
        r = sorted_rows(ref[key])
        assert g.shape == r.shape and np.array_equal(g.view(np.uint32), r.view(np.uint32)), dim
