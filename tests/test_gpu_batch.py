"""Batching form: a batch of clouds gives, per cloud, exactly the diagrams
of separate rips_persistence calls (and of the oracle)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from golden_util import golden_cases, load_golden, sorted_rows

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


def _same(a, b):
    a = np.asarray(a.cpu() if isinstance(a, torch.Tensor) else a, dtype=np.float32).reshape(-1, 2)
    b = np.asarray(b.cpu() if isinstance(b, torch.Tensor) else b, dtype=np.float32).reshape(-1, 2)
    return a.shape == b.shape and np.array_equal(_bits(a), _bits(b))


def test_batch_of_golden_clouds_equals_single_calls():
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import rips_persistence_batch
    names = golden_cases()
    clouds, ts, dims = [], [], []
    for nm in names:
        z, meta = load_golden(nm)
        clouds.append(z["points"])
        ts.append(float(z["t"]))
        dims.append(meta["max_dim"])
    res = rips_persistence_batch(clouds, ts, dims)
    assert len(res) == len(names)
    for nm, p, t, md, r in zip(names, clouds, ts, dims, res):
        assert not isinstance(r, Exception), (nm, r)
        single = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=md)
        assert len(r) == md + 1, nm
        for dim in range(md + 1):
            assert _same(r[dim], single[dim]), (nm, dim)


def test_mixed_dims_and_sizes_against_oracle():
    from flashph_b200.batch import rips_persistence_batch
    rng = np.random.default_rng(11)
    clouds, ts, dims = [], [], []
    for c in range(24):
        n = int(rng.integers(2, 400))
        d = int(rng.choice([2, 3, 8, 32]))
        clouds.append(rng.standard_normal((n, d)).astype(np.float32))
        ts.append(float({2: 0.5, 3: 0.9, 8: 2.6, 32: 6.8}[d]))
        dims.append(int(rng.choice([0, 1, 2])))
    res = rips_persistence_batch(clouds, ts, dims)
    for p, t, md, r in zip(clouds, ts, dims, res):
        ref = oracle.run(p, t, md, fused=True)
        assert _same(r[0], ref["h0"])
        if md >= 1:
            assert _same(r[1], ref["h1"])
        if md >= 2:
            assert _same(sorted_rows(r[2].cpu().numpy()), sorted_rows(ref["h2"]))


def test_per_cloud_errors_do_not_stop_the_batch():
    from flashph_b200.batch import rips_persistence_batch
    rng = np.random.default_rng(3)
    good = rng.standard_normal((50, 3)).astype(np.float32)
    dense = rng.standard_normal((300, 3)).astype(np.float32) * 0.01
    res = rips_persistence_batch([good, good, np.zeros((0, 3), np.float32), good[:1], dense],
                                 [1.0, -1.0, 1.0, 1.0, 1.0], [1, 1, 2, 1, 1], max_triangles=100_000)
    assert not isinstance(res[0], Exception)
    assert isinstance(res[1], ValueError) and "non-negative" in str(res[1])
    assert [x.shape for x in res[2]] == [(0, 2)] * 3
    assert res[3][0].tolist() == [[0.0, float("inf")]]
    assert isinstance(res[4], ValueError) and "max_triangles" in str(res[4])


def test_auto_threshold_batch_equals_single():
    from flashph_b200 import auto_threshold
    from flashph_b200.batch import auto_threshold_batch
    rng = np.random.default_rng(5)
    clouds = [rng.standard_normal((int(n), int(d))).astype(np.float32)
              for n, d in zip(rng.integers(2, 700, 12), rng.choice([3, 8, 32], 12))]
    clouds.append(np.zeros((1, 3), np.float32))
    got = auto_threshold_batch(clouds, k=20, percentile=95.0)
    want = [auto_threshold(torch.from_numpy(c).cuda(), k=20, percentile=95.0) for c in clouds]
    assert got == want
    # and within float32 rounding of a float64 restatement
    for c, g in zip(clouds[:-1], got[:-1]):
        d2 = ((c[:, None, :].astype(np.float64) - c[None, :, :]) ** 2).sum(-1)
        np.fill_diagonal(d2, np.inf)
        k = max(1, min(20, c.shape[0] - 1))
        kth = np.sqrt(np.sort(d2, axis=1)[:, k - 1])
        assert abs(g - np.quantile(kth, 0.95)) <= 1e-5 * max(1.0, abs(g))


def test_large_clouds_take_the_native_route_and_match_single_calls():
    """Clouds on both sides of NATIVE_MIN_POINTS (native calls on worker
    streams, and the union pipeline), CUDA and host inputs, and a large cloud
    over the triangle cap: every result equals its single call or the
    reference's error."""
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import NATIVE_MIN_POINTS, rips_persistence_batch
    rng = np.random.default_rng(17)
    sizes = [NATIVE_MIN_POINTS - 1, NATIVE_MIN_POINTS, 1500, 300, 2600, 64]
    clouds, ts, dims = [], [], []
    for k, n in enumerate(sizes):
        d = [3, 8, 10][k % 3]
        clouds.append(rng.standard_normal((n, d)).astype(np.float32))
        ts.append({3: 0.35, 8: 1.5, 10: 1.9}[d])
        dims.append(2 if k % 2 == 0 else 1)
    clouds[4] = torch.from_numpy(clouds[4]).cuda()  # a device input among host ones
    dense = (rng.standard_normal((1200, 3)) * 0.05).astype(np.float32)
    clouds.append(dense)
    ts.append(10.0)
    dims.append(1)
    res = rips_persistence_batch(clouds, ts, dims, max_triangles=5_000_000)
    assert isinstance(res[-1], ValueError) and "max_triangles=5000000" in str(res[-1])
    for p, t, md, r in zip(clouds[:-1], ts[:-1], dims[:-1], res[:-1]):
        assert not isinstance(r, Exception), r
        x = p if isinstance(p, torch.Tensor) else torch.from_numpy(p).cuda()
        single = rips_persistence(x, t, max_dim=md)
        assert len(r) == md + 1
        for dim in range(md + 1):
            assert r[dim].device.type == "cuda"
            assert _same(r[dim], single[dim]), (p.shape, dim)


def _mixed_clouds(seed=23):
    """Clouds of every kind the batch must keep apart: H0-only, H1, H2, n = 2,
    a cloud over the triangle limit, one over the tetrahedron limit, both edge
    kernels' dimensions."""
    rng = np.random.default_rng(seed)
    clouds, ts, dims = [], [], []
    for k in range(18):
        n = int(rng.integers(2, 700))
        d = int(rng.choice([2, 3, 8, 32]))
        clouds.append(rng.standard_normal((n, d)).astype(np.float32))
        ts.append(float({2: 0.6, 3: 0.9, 8: 2.6, 32: 6.8}[d]))
        dims.append(int(rng.choice([0, 1, 2])))
    clouds.append((rng.standard_normal((500, 3)) * 0.05).astype(np.float32))  # over max_triangles
    ts.append(10.0)
    dims.append(1)
    clouds.append((rng.standard_normal((120, 4)) * 0.3).astype(np.float32))  # complete: C(120,4) > max_tetrahedra
    ts.append(2.5)
    dims.append(2)
    return clouds, ts, dims


def test_native_batch_equals_staged_batch_and_single_calls(monkeypatch):
    """ph_rips_persistence_batch (one library call for the whole union)
    against the stage-by-stage union and against single calls, bit for bit;
    per-cloud limit errors carry the reference's texts."""
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import rips_persistence_batch
    clouds, ts, dims = _mixed_clouds()
    native = rips_persistence_batch(clouds, ts, dims, max_triangles=2_000_000, max_tetrahedra=1_000_000)
    monkeypatch.setenv("FLASHPH_BATCH", "staged")
    staged = rips_persistence_batch(clouds, ts, dims, max_triangles=2_000_000, max_tetrahedra=1_000_000)
    monkeypatch.delenv("FLASHPH_BATCH")
    assert isinstance(native[-2], ValueError) and "max_triangles=2000000" in str(native[-2])
    assert isinstance(native[-1], ValueError) and "max_tetrahedra=1000000" in str(native[-1])
    for c, (p, t, md, a, b) in enumerate(zip(clouds, ts, dims, native, staged)):
        if isinstance(a, Exception):
            assert isinstance(b, ValueError) and str(a) == str(b), c
            with pytest.raises(ValueError) as ex:
                _single_with_limits(p, t, md)
            assert str(ex.value) == str(a), c
            continue
        single = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=md)
        assert len(a) == len(b) == md + 1, c
        for dim in range(md + 1):
            assert _same(a[dim], b[dim]) and _same(a[dim], single[dim]), (c, dim)


def _single_with_limits(p, t, md):
    """rips_persistence of one cloud with the limits of the batch above."""
    from flashph_b200.persistence import _compute_native
    x = torch.from_numpy(p).cuda()
    return _compute_native(x, t, md, x.device, 2_000_000, 1_000_000)


def test_exact_triangle_precount_under_and_over_the_limit():
    """Clouds with more edges than the triangle bound allows for max_triangles
    are counted exactly before the per-edge pass: one of them under the limit
    (its diagrams must equal a single call's), one over it (the single call's
    ValueError text, with the exact count), beside clouds too sparse to be
    counted early."""
    from flashph_b200.batch import rips_persistence_batch
    from flashph_b200.persistence import _compute_native
    rng = np.random.default_rng(41)
    cap = 200_000  # the bound lets clouds of up to ~5.6K edges through uncounted
    clouds = [rng.standard_normal((1000, 3)).astype(np.float32),          # counted early, under the limit
              (rng.standard_normal((400, 3)) * 0.05).astype(np.float32),  # complete: C(400,3) over it
              rng.standard_normal((300, 8)).astype(np.float32),
              rng.standard_normal((64, 2)).astype(np.float32)]
    ts = [0.6, 10.0, 2.2, 0.6]  # cloud 0: 9,305 edges and 40,242 triangles (oracle)
    dims = [1, 1, 1, 1]
    res = rips_persistence_batch(clouds, ts, dims, max_triangles=cap)
    for c, (p, t, md, r) in enumerate(zip(clouds, ts, dims, res)):
        x = torch.from_numpy(p).cuda()
        try:
            single = _compute_native(x, t, md, x.device, cap, 10_000_000)
        except ValueError as ex:
            assert isinstance(r, ValueError) and str(r) == str(ex), c
            continue
        assert not isinstance(r, Exception), (c, r)
        for dim in range(md + 1):
            assert _same(r[dim], single[dim]), (c, dim)
    assert isinstance(res[1], ValueError) and "Triangle count 10586800 exceeds" in str(res[1])
    assert not isinstance(res[0], Exception)


def test_batch_split_by_the_simplex_budget(monkeypatch):
    """A budget small enough to split every chunk: the library reports the
    per-cloud counts, the batch is packed again, results are unchanged."""
    from flashph_b200 import batch as B
    clouds, ts, dims = _mixed_clouds(seed=29)
    whole = B.rips_persistence_batch(clouds, ts, dims, max_triangles=2_000_000, max_tetrahedra=1_000_000)
    monkeypatch.setattr(B, "_BATCH_SIMPLICES", 30_000)
    split = B.rips_persistence_batch(clouds, ts, dims, max_triangles=2_000_000, max_tetrahedra=1_000_000)
    for a, b in zip(whole, split):
        if isinstance(a, Exception):
            assert str(a) == str(b)
            continue
        for x, y in zip(a, b):
            assert _same(x, y)


def test_union_of_dense_clouds_matches_single_calls():
    """Dense clouds of the batching configuration (noisy rotated Clifford tori
    and Gaussian clouds at the 95th percentile of 20-NN distances, 800-1900
    points) in one union: several clouds with millions of triangle rows, whose
    working-column bitmaps are windows of one cloud's row range. Each against
    its single call, bit for bit."""
    import bench
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import auto_threshold_batch, rips_persistence_batch
    rng = np.random.default_rng(31)
    clouds = []
    for k, (n, d) in enumerate([(1100, 8), (1900, 3), (800, 32), (1500, 8), (1300, 3)]):
        clouds.append(rng.standard_normal((n, d)).astype(np.float32) if k % 2 == 0
                      else bench.clifford_cloud(n, d, rng))
    ts = auto_threshold_batch(clouds, k=20, percentile=95.0)
    res = rips_persistence_batch(clouds, ts, 1)
    for p, t, r in zip(clouds, ts, res):
        single = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=1)
        assert not isinstance(r, Exception), r
        assert _same(r[0], single[0]) and _same(r[1], single[1])
