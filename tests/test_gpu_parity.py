"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

The oracle runs with the fused dist^2 chain (the arithmetic of the
reference's compiled GPU kernel) and correctly rounded square roots (torch
on CUDA). Edges, their order, the forest, the H0 rows and the H1 rows (in
the reference's exact row order) must be bit-identical; H2, which the
reference delegates to giotto-ph, is compared as a multiset of rows.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from golden_util import golden_cases, load_golden, sorted_rows

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _fp(pts):
    return torch.from_numpy(np.ascontiguousarray(pts)).to(DEV)


def _bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


def _same_rows(a, b):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    return a.shape == b.shape and np.array_equal(_bits(a), _bits(b))


@pytest.mark.parametrize("name", golden_cases())
def test_pipeline_matches_oracle(name):
    from flashph_b200 import rips_persistence
    from flashph_b200.rips import rips_filtration
    z, meta = load_golden(name)
    pts, t, md = z["points"], float(z["t"]), meta["max_dim"]
    ref = oracle.run(pts, t, md, fused=True)
    if pts.shape[0] >= 2:
        f = rips_filtration(_fp(pts), t)
        assert f.edge_i.shape[0] == ref["E"]
        assert np.array_equal(f.edge_i.cpu().numpy(), ref["edge_i"])
        assert np.array_equal(f.edge_j.cpu().numpy(), ref["edge_j"])
        assert np.array_equal(_bits(f.edge_dist_sq.cpu().numpy()), _bits(ref["edge_dsq"]))
    dg = rips_persistence(_fp(pts), t, max_dim=md)
    assert len(dg) == md + 1
    assert all(d.device.type == "cuda" and d.dtype == torch.float32 for d in dg)
    assert _same_rows(dg[0].cpu().numpy(), ref["h0"].reshape(-1, 2)), "H0"
    if md >= 1:
        assert _same_rows(dg[1].cpu().numpy(), ref["h1"].reshape(-1, 2)), "H1 rows/order"
    if md >= 2:
        assert _same_rows(sorted_rows(dg[2].cpu().numpy()), sorted_rows(ref["h2"])), "H2 multiset"


@pytest.mark.parametrize("name", [c for c in golden_cases() if load_golden(c)[1]["max_dim"] >= 1])
def test_h1_pairs_and_classes_match_oracle(name):
    """Apparent/residual/essential classification and pivots, bit-exact."""
    from flashph_b200.boruvka import boruvka_mask
    from flashph_b200.cohomology import h1_diagram
    from flashph_b200.rips import edge_filtration_values, rips_filtration
    z, meta = load_golden(name)
    pts, t = z["points"], float(z["t"])
    if pts.shape[0] < 2:
        return
    ref = oracle.run(pts, t, 1, fused=True)
    f = rips_filtration(_fp(pts), t)
    ef = edge_filtration_values(f.edge_dist_sq)
    mst, comp, (ncomp, st) = boruvka_mask(f.edge_i, f.edge_j, pts.shape[0])
    assert int(st.item()) == 0
    assert np.array_equal(np.nonzero(mst.cpu().numpy())[0], ref["mst_idx"])
    assert int(ncomp.item()) == ref["n_components"]
    rows, tris, red, info = h1_diagram(f, ef, mst)
    assert tris.T == ref["T"]
    if ref["T"] == 0:  # the reference builds the rows directly; no pairs
        assert np.array_equal(_bits(rows.cpu().numpy()), _bits(ref["h1"]))
        return
    state = red.state.cpu().numpy()
    piv = red.piv.cpu().numpy()
    E = ref["E"]
    assert int((state == 1).sum()) == ref["n_apparent"]
    assert int((state == 0).sum()) == len(ref["mst_idx"])
    # the reference's residual count includes columns without cofacets (and is
    # not computed at all when there are no triangles)
    if ref["T"] > 0:
        assert int((state != 0).sum()) - int((state == 1).sum()) == ref["residual"]
    assert int(info[0]) <= ref["residual"]
    # every pair of the oracle appears with the same pivot
    for b, dth in zip(ref["ap_births"], ref["ap_deaths"]):
        assert state[b] == 1 and piv[b] == dth
    for b, dth in zip(ref["res_births"], ref["res_deaths"]):
        assert state[b] == 2 and piv[b] == dth
    ess = set(ref["ess_births"].tolist())
    assert ess == set(np.nonzero(state == 3)[0].tolist())
    # pivots of all nonzero columns equal the oracle's H1 pivot set
    gpu_piv = np.sort(piv[(state == 1) | (state == 2)])
    assert np.array_equal(gpu_piv, np.sort(ref["h1_all_pivots"]))
    assert E == f.edge_i.shape[0]


def test_numpy_and_cpu_inputs():
    from flashph_b200 import rips_persistence
    rng = np.random.default_rng(0)
    pts = rng.standard_normal((60, 3)).astype(np.float32)
    a = rips_persistence(pts, 1.2)
    assert a[0].device.type == "cuda"
    b = rips_persistence(torch.from_numpy(pts), 1.2)
    assert b[0].device.type == "cpu"
    for x, y in zip(a, b):
        assert torch.equal(x.cpu(), y)


def test_edge_cases_on_device():
    from flashph_b200 import rips_persistence
    d = rips_persistence(torch.empty(0, 3, device=DEV), 1.0, max_dim=2)
    assert len(d) == 3 and all(x.shape == (0, 2) and x.device.type == "cuda" for x in d)
    d = rips_persistence(torch.tensor([[1.0, 2.0, 3.0]], device=DEV), 1.0, max_dim=2)
    assert d[0].tolist() == [[0.0, float("inf")]]
    d = rips_persistence(torch.randn(50, 3, device=DEV), 1e-10, max_dim=1)
    assert d[1].shape == (0, 2) and d[0].shape == (50, 2)
    assert torch.isinf(d[0][:, 1]).all()


def test_circle_betti():
    from flashph_b200 import RipsComplex
    th = torch.linspace(0, 2 * 3.14159265, 21)[:20]
    pts = torch.stack([torch.cos(th), torch.sin(th)], 1).to(DEV)
    rc = RipsComplex(pts, 0.5)
    rc.compute_persistence(max_dim=1)
    assert rc.betti_numbers() == [1, 1]
    assert rc.persistent_betti_numbers(0.0, float("inf")) == [0, 0]


def test_clifford_torus_significant_bars():
    """Known answer (reference test_persistence.py:541-570): 1 component,
    2 H1 and 1 H2 bars with persistence > 0.4."""
    from flashph_b200 import rips_persistence
    z, _ = load_golden("clifford200_t14_h2")
    dg = rips_persistence(_fp(z["points"]), 1.4, max_dim=2)
    assert int(torch.isinf(dg[0][:, 1]).sum()) == 1
    for dim, want in ((1, 2), (2, 1)):
        fin = dg[dim][torch.isfinite(dg[dim][:, 1])]
        assert int(((fin[:, 1] - fin[:, 0]) > 0.4).sum()) == want


def test_ripscomplex_matches_flat_api():
    from flashph_b200 import RipsComplex, rips_persistence
    pts = _fp(np.random.default_rng(42).standard_normal((50, 2)).astype(np.float32))
    rc = RipsComplex(pts, 3.0)
    rc.compute_persistence(max_dim=1)
    flat = rips_persistence(pts, 3.0)
    for dim in range(2):
        iv = rc.persistence_intervals_in_dimension(dim)
        assert iv.dtype == np.float64
        np.testing.assert_allclose(iv, flat[dim].cpu().numpy().astype(np.float64), atol=1e-6)
    assert rc.persistence_intervals_in_dimension(5).shape == (0, 2)
    res = rc.persistence(max_dim=1)
    keys = [(d, b, de) for d, (b, de) in res]
    assert keys == sorted(keys) and len(keys) > 0


def test_repeat_calls_are_deterministic():
    from flashph_b200 import rips_persistence
    z, _ = load_golden("n500_d10_t28_h2")
    a = rips_persistence(_fp(z["points"]), 2.8, max_dim=2)
    b = rips_persistence(_fp(z["points"]), 2.8, max_dim=2)
    assert _same_rows(a[0].cpu(), b[0].cpu()) and _same_rows(a[1].cpu(), b[1].cpu())
    assert _same_rows(sorted_rows(a[2].cpu()), sorted_rows(b[2].cpu()))


def test_colex_collisions_follow_emission_order():
    from flashph_b200.rips import rips_filtration
    from test_cpu_host import colex_collision_cloud, emission_key
    pts, pairs = colex_collision_cloud(extra=True)
    f = rips_filtration(_fp(pts), 1.5)
    got = list(zip(f.edge_i.cpu().tolist(), f.edge_j.cpu().tolist()))
    assert got == sorted(pairs, key=lambda p: emission_key(*p))


def test_twenty_k_matches_oracle():
    """The benchmark workload (n=20000, d=10, t=1.4, H0-H2) against the oracle."""
    from flashph_b200 import rips_persistence
    pts = np.random.default_rng(42).standard_normal((20000, 10)).astype(np.float32)
    ref = oracle.run(pts, 1.4, 2, fused=True)
    dg = rips_persistence(_fp(pts), 1.4, max_dim=2)
    assert _same_rows(dg[0].cpu().numpy(), ref["h0"])
    assert _same_rows(dg[1].cpu().numpy(), ref["h1"])
    assert _same_rows(sorted_rows(dg[2].cpu().numpy()), sorted_rows(ref["h2"]))


@pytest.mark.parametrize("name", golden_cases())
def test_native_pipeline_equals_staged(name, monkeypatch):
    """ph_rips_persistence (one native call) and the stage-by-stage Python
    path give the same diagrams, bit for bit and in the same row order."""
    from flashph_b200 import rips_persistence
    z, meta = load_golden(name)
    pts, t, md = z["points"], float(z["t"]), meta["max_dim"]
    native = rips_persistence(_fp(pts), t, max_dim=md)
    monkeypatch.setenv("FLASHPH_PIPELINE", "staged")
    staged = rips_persistence(_fp(pts), t, max_dim=md)
    assert len(native) == len(staged)
    for a, b in zip(native, staged):
        assert _bits(a.cpu().numpy()).shape == _bits(b.cpu().numpy()).shape
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b.cpu().numpy()))


def test_native_pipeline_host_arrays_and_limits():
    from flashph_b200 import rips_persistence
    rng = np.random.default_rng(21)
    pts = rng.standard_normal((3000, 10)).astype(np.float32)
    dev = rips_persistence(torch.from_numpy(pts).cuda(), 1.6, max_dim=2)
    host = rips_persistence(torch.from_numpy(pts), 1.6, max_dim=2)  # CPU in, CPU out
    for a, b in zip(dev, host):
        assert b.device.type == "cpu"
        assert np.array_equal(_bits(a.cpu().numpy()), _bits(b.numpy()))
    dense = rng.standard_normal((400, 3)).astype(np.float32)  # complete graph: C(400, 3) > 10^7 triangles
    with pytest.raises(ValueError, match="exceeds max_triangles=10000000"):
        rips_persistence(torch.from_numpy(dense).cuda(), 100.0, max_dim=1)


@pytest.mark.parametrize("n", [450, 500])
def test_dense_columns_in_global_bitmaps_match_oracle(n):
    """Dense H1 (d = 50 at the 30th percentile of distances): about 10^6
    triangle rows, more than a warp's shared bitmap holds, and working columns
    of 9K-40K entries (the oracle's col_max), longer than the shared list
    buffers: columns become bitmaps in global memory. Bit for bit against the
    oracle."""
    import oracle
    from flashph_b200 import rips_persistence
    rng = np.random.default_rng(5)
    if n == 500:
        rng.standard_normal((450, 50))  # the same stream as the probe that sized these cases
    p = rng.standard_normal((n, 50)).astype(np.float32)
    dd = np.sqrt(((p[:, None, :].astype(np.float64) - p[None]) ** 2).sum(-1))
    t = float(np.quantile(dd[np.triu_indices(n, 1)], 0.30))
    ref = oracle.run(p, t, 1, fused=True)
    assert ref["T"] > 196_608 and ref["col_max"] > 6144
    got = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=1)
    assert _same_rows(got[0].cpu(), ref["h0"])
    assert _same_rows(got[1].cpu(), ref["h1"])


def test_h2_with_list_columns_matches_oracle():
    """H2 with 363K tetrahedron rows: more than a warp's shared bitmap holds,
    so the H2 working columns are sorted lists in shared memory (the
    broadcast-rank XOR for short added columns); H1 of the same cloud uses
    the shared bitmaps. H0-H2 against the oracle."""
    import oracle
    from flashph_b200 import rips_persistence
    p = np.random.default_rng(9).standard_normal((200, 20)).astype(np.float32)
    dd = np.sqrt(((p[:, None, :].astype(np.float64) - p[None]) ** 2).sum(-1))
    t = float(np.quantile(dd[np.triu_indices(200, 1)], 0.25))
    ref = oracle.run(p, t, 2, fused=True)
    assert ref["Q"] > 196_608 and ref["T"] < 196_608
    got = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=2)
    assert _same_rows(got[0].cpu(), ref["h0"])
    assert _same_rows(got[1].cpu(), ref["h1"])
    assert _same_rows(sorted_rows(got[2].cpu().numpy()), sorted_rows(ref["h2"]))


def test_dense_h1_with_ten_million_rows_matches_oracle():
    """A batching-configuration-sized dense cloud (n = 1898, d = 8, t = 2.701:
    202,737 edges, 9,776,543 triangle rows, working columns up to 127,972
    entries): the global bitmaps span ~9.8M rows and are scanned through their
    shared-memory summary (one bit per 1024 rows). Bit for bit against the
    oracle."""
    import oracle
    from flashph_b200 import rips_persistence
    p = np.random.default_rng(2).standard_normal((1898, 8)).astype(np.float32)
    ref = oracle.run(p, 2.701, 1, fused=True)
    assert ref["T"] > 9_000_000 and ref["col_max"] > 100_000
    got = rips_persistence(torch.from_numpy(p).cuda(), 2.701, max_dim=1)
    assert _same_rows(got[0].cpu(), ref["h0"])
    assert _same_rows(got[1].cpu(), ref["h1"])


def test_dense_h2_with_million_tetrahedron_rows_matches_oracle():
    """H2 of a d = 50 cloud with millions of tetrahedron rows (the serving
    stream's dense H2 requests): H2 working columns become global bitmaps
    with a summary. H0-H2 against the oracle (H2 as a multiset)."""
    import oracle
    from flashph_b200 import rips_persistence
    p = np.random.default_rng(4).standard_normal((240, 50)).astype(np.float32)
    dd = np.sqrt(((p[:, None, :].astype(np.float64) - p[None]) ** 2).sum(-1))
    t = float(np.quantile(dd[np.triu_indices(240, 1)], 0.30))
    ref = oracle.run(p, t, 2, fused=True)
    assert ref["Q"] > 1_000_000
    got = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=2)
    assert _same_rows(got[0].cpu(), ref["h0"])
    assert _same_rows(got[1].cpu(), ref["h1"])
    assert _same_rows(sorted_rows(got[2].cpu().numpy()), sorted_rows(ref["h2"]))
