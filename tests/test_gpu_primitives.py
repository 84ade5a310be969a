"""GPU checks of the filtration-sort and adjacency entry points on random
inputs at tile-boundary sizes, against numpy stable sorts."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _random_edges(E, n, seed):
    rng = np.random.default_rng(seed)
    # distinct pairs i < j
    flat = rng.choice(n * (n - 1) // 2, size=E, replace=False)
    j = np.floor((1 + np.sqrt(1 + 8 * flat.astype(np.float64))) / 2).astype(np.int64)
    j = np.where(j * (j - 1) // 2 > flat, j - 1, j)
    j = np.where((j + 1) * j // 2 <= flat, j + 1, j)
    i = flat - j * (j - 1) // 2
    assert np.all((0 <= i) & (i < j) & (j < n))
    # few distinct lengths so that dist^2 ties are frequent
    dsq = rng.integers(0, 50, size=E).astype(np.float32) / np.float32(7.0)
    return i.astype(np.int32), j.astype(np.int32), dsq


@pytest.mark.parametrize("E", [1, 2, 5, 17, 4095, 4096, 4097, 70000, 98304, 98305, 1 << 20])
def test_edges_sort_matches_numpy(E):
    from flashph_b200.rips import sort_edges
    n = 50000
    ei, ej, ed = _random_edges(E, n, E)
    key = (ed.view(np.uint32).astype(np.uint64) << np.uint64(32)) | (
        (ej.astype(np.uint64) * (ej.astype(np.uint64) - np.uint64(1)) // np.uint64(2) + ei.astype(np.uint64))
        & np.uint64(0xFFFFFFFF))
    order = np.argsort(key, kind="stable")
    oi, oj, od = sort_edges(torch.from_numpy(ei).cuda(), torch.from_numpy(ej).cuda(),
                            torch.from_numpy(ed).cuda(), n)
    assert np.array_equal(oi.cpu().numpy(), ei[order])
    assert np.array_equal(oj.cpu().numpy(), ej[order])
    assert np.array_equal(od.cpu().numpy().view(np.uint32), ed[order].view(np.uint32))


@pytest.mark.parametrize("E,n", [(1, 2), (100, 1000), (5000, 300), (200000, 100000)])
def test_vertex_csr_matches_numpy(E, n):
    from flashph_b200.rips import vertex_csr
    ei, ej, _ = _random_edges(E, n, 7 + E)
    ptr, idx, rank = vertex_csr(torch.from_numpy(ei).cuda(), torch.from_numpy(ej).cuda(), n)
    src = np.concatenate([ei, ej]).astype(np.int64)
    dst = np.concatenate([ej, ei]).astype(np.int64)
    rk = np.concatenate([np.arange(E), np.arange(E)])
    o = np.argsort(src * n + dst, kind="stable")
    want_ptr = np.zeros(n + 1, np.int64)
    np.add.at(want_ptr, src + 1, 1)
    want_ptr = np.cumsum(want_ptr)
    assert np.array_equal(ptr.cpu().numpy(), want_ptr)
    assert np.array_equal(idx.cpu().numpy(), dst[o])
    assert np.array_equal(rank.cpu().numpy(), rk[o])


def test_launch_counter_advances():
    from flashph_b200 import _lib
    from flashph_b200.rips import sort_edges
    ei, ej, ed = _random_edges(1000, 100, 3)
    before = _lib.launch_count()
    sort_edges(torch.from_numpy(ei).cuda(), torch.from_numpy(ej).cuda(), torch.from_numpy(ed).cuda(), 100)
    torch.cuda.synchronize()
    assert _lib.launch_count() > before


@pytest.mark.parametrize("n,d,t", [(500, 3, 0.3), (2000, 4, 0.9), (1500, 10, 3.0), (800, 2, 5.0), (3, 2, 9.0)])
def test_triangle_total_equals_per_edge_counts(n, d, t):
    """ph_triangles_total (rank-free, bitmap) equals the sum of the per-edge
    triangle counts on sparse, dense and complete graphs."""
    from flashph_b200 import _lib as L
    from flashph_b200.cohomology import count_triangles
    from flashph_b200.rips import rips_filtration
    x = torch.from_numpy(np.random.default_rng(n + d).standard_normal((n, d)).astype(np.float32)).cuda()
    f = rips_filtration(x, t)
    E = f.edge_i.shape[0]
    want = int(count_triangles(f)[E].item())
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    nxt = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("ph_triangles_total", f.vert_adj_ptr.data_ptr(), f.vert_adj_idx.data_ptr(), n, tot.data_ptr(),
           nxt.data_ptr(), L.stream_handle(x.device))
    assert int(tot.item()) == want


@pytest.mark.parametrize("n,d,t", [(500, 3, 0.3), (1500, 10, 3.0), (3, 2, 9.0)])
def test_batch_triangle_totals_per_cloud(n, d, t):
    """ph_batch_triangles_total over a union of three copies of one graph
    (vertices offset by n and 2n): each wanted cloud gets the single graph's
    total, the cloud not wanted gets 0."""
    from flashph_b200 import _lib as L
    from flashph_b200.cohomology import count_triangles
    from flashph_b200.rips import rips_filtration, vertex_csr
    x = torch.from_numpy(np.random.default_rng(n + d).standard_normal((n, d)).astype(np.float32)).cuda()
    f = rips_filtration(x, t)
    E = f.edge_i.shape[0]
    want_total = int(count_triangles(f)[E].item())
    ei = torch.cat([f.edge_i + k * n for k in range(3)]).contiguous()
    ej = torch.cat([f.edge_j + k * n for k in range(3)]).contiguous()
    ptr, idx, _ = vertex_csr(ei, ej, 3 * n)
    vcloud = torch.arange(3 * n, device="cuda", dtype=torch.int32) // n
    want = torch.tensor([1, 0, 1], dtype=torch.uint8, device="cuda")
    per = torch.full((3,), 7, dtype=torch.int64, device="cuda")
    nxt = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("ph_batch_triangles_total", ptr.data_ptr(), idx.data_ptr(), 3 * n, vcloud.data_ptr(), want.data_ptr(), 3,
           per.data_ptr(), nxt.data_ptr(), L.stream_handle(x.device))
    assert per.cpu().tolist() == [want_total, 0, want_total]


def test_dense_call_over_the_triangle_limit_reports_the_exact_count():
    from flashph_b200 import rips_persistence
    pts = np.random.default_rng(5).standard_normal((3000, 3)).astype(np.float32)
    with pytest.raises(ValueError, match="Triangle count 4495501000 exceeds max_triangles=10000000"):
        rips_persistence(torch.from_numpy(pts).cuda(), 1e3, max_dim=1)  # complete graph: C(3000, 3)


def _kruskal(ei, ej, n):
    """Forest mask and smallest-vertex labels by Kruskal over the positions."""
    parent = list(range(n))

    def find(v):
        while parent[v] != v:
            parent[v] = parent[parent[v]]
            v = parent[v]
        return v

    mask = np.zeros(len(ei), np.uint8)
    for e, (a, b) in enumerate(zip(ei.tolist(), ej.tolist())):
        ra, rb = find(a), find(b)
        if ra != rb:
            mask[e] = 1
            parent[max(ra, rb)] = min(ra, rb)
    comp = np.array([find(v) for v in range(n)], np.int32)
    return mask, comp


@pytest.mark.parametrize("n,E", [(2, 1), (300, 200), (1000, 3000), (5000, 12000), (20000, 30000),
                                 (29000, 80000), (120000, 400000), (700000, 900000)])
def test_forest_cluster_and_grid_forms_match_kruskal(n, E):
    """Every form of the forest kernel (one block for tiny graphs, a thread
    block cluster with the vertices in distributed shared memory up to about
    450K vertices, a cooperative grid above) against Kruskal, on random
    multigraphs with self-loops, repeated pairs, long paths and many
    components."""
    from flashph_b200.boruvka import boruvka_mask
    rng = np.random.default_rng(n + E)
    ei = rng.integers(0, n, E).astype(np.int32)
    ej = rng.integers(0, n, E).astype(np.int32)
    if E > 10:
        k = E // 10  # a long path in scrambled rank order
        ei[:k] = np.arange(k) % n
        ej[:k] = (np.arange(k) + 1) % n
        perm = rng.permutation(E)
        ei, ej = ei[perm], ej[perm]
        ej[::97] = ei[::97]  # self-loops
    ref_mask, ref_comp = _kruskal(ei, ej, n)
    mask, comp, (ncomp, status) = boruvka_mask(torch.from_numpy(ei).cuda(), torch.from_numpy(ej).cuda(), n)
    assert int(status.item()) == 0
    assert np.array_equal(mask.cpu().numpy(), ref_mask)
    assert np.array_equal(comp.cpu().numpy(), ref_comp)
    assert int(ncomp.item()) == int((ref_comp == np.arange(n)).sum())


@pytest.mark.parametrize("E", [1, 2047, 2048, 2049, 1 << 20, (1 << 22) + 5])
def test_h0_rows_through_both_scan_forms(E):
    """H0 rows place forest edge e at the exclusive prefix count of the mask:
    the single-launch scan (up to 4M entries) and the three-launch one
    (above) against numpy, at tile-boundary sizes."""
    from flashph_b200.boruvka import h0_rows
    rng = np.random.default_rng(E)
    n = E + 7
    mask = (rng.random(E) < 0.3).astype(np.uint8)
    filt = np.sort(rng.random(E).astype(np.float32))
    rows = h0_rows(torch.from_numpy(filt).cuda(), torch.from_numpy(mask).cuda(), n).cpu().numpy()
    k = int(mask.sum())
    assert rows.shape == (n, 2)
    assert np.all(rows[:, 0] == 0)
    assert np.array_equal(rows[:k, 1], filt[mask == 1])
    assert np.all(np.isinf(rows[k:, 1]))


@pytest.mark.parametrize("seed", [0, 1])
def test_cofacet_rows_without_sort_equal_the_sorted_csr(seed):
    """ph_cofacet_rows3 (entries scattered into rows whose lengths are known,
    then each row sorted in shared memory) against ph_cofacet_csr (stable
    radix sort by face), on triangles with random faces and a few hub faces
    in thousands of triangles (rows sorted by a warp, by a block, and rows of
    one entry); identical offsets and rows, and the longest row reported."""
    from flashph_b200 import _lib as L
    rng = np.random.default_rng(seed)
    E, T = 6000, 60000
    f = rng.integers(0, E, size=(T, 3)).astype(np.int32)
    hubs = np.array([7, 4000, 5999], dtype=np.int32)
    for h, cnt in zip(hubs, (3000, 1500, 40)):
        idx = rng.choice(T, size=cnt, replace=False)
        f[idx, rng.integers(0, 3, size=cnt)] = h
    f0, f1, f2 = (torch.from_numpy(np.ascontiguousarray(f[:, q])).cuda() for q in range(3))
    counts = np.bincount(f.reshape(-1), minlength=E).astype(np.int64)
    off = np.zeros(E + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    off_d = torch.from_numpy(off).cuda()
    s = torch.cuda.current_stream().cuda_stream
    mx = torch.zeros(1, dtype=torch.int64, device="cuda")
    L.call("ph_max_count", off_d.data_ptr(), E, mx.data_ptr(), s)
    assert int(mx.item()) == int(counts.max()) > 2048
    want_off = torch.empty(E + 1, dtype=torch.int32, device="cuda")
    want = torch.empty(3 * T, dtype=torch.int32, device="cuda")
    nb = L.query("ph_cofacet_csr_workspace_bytes", T, 3)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    L.call("ph_cofacet_csr", None, f0.data_ptr(), f1.data_ptr(), f2.data_ptr(), 3, T, E, 100000,
           want_off.data_ptr(), want.data_ptr(), ws.data_ptr(), nb, s)
    got_off = torch.empty(E + 1, dtype=torch.int32, device="cuda")
    got = torch.empty(3 * T, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    nb3 = L.query("ph_cofacet_rows3_workspace_bytes", E)
    ws3 = torch.empty(nb3, dtype=torch.uint8, device="cuda")
    L.call("ph_cofacet_rows3", f0.data_ptr(), f1.data_ptr(), f2.data_ptr(), T, E, 100000, off_d.data_ptr(),
           int(mx.item()), got_off.data_ptr(), got.data_ptr(), st.data_ptr(), ws3.data_ptr(), nb3, s)
    assert int(st.item()) == 0
    assert torch.equal(got_off, want_off)
    assert torch.equal(got, want)
    # a longest row beyond the in-shared-memory sort is refused before any work
    too_long = int(L.lib().ph_cofacet_rows3_max_row()) + 1
    rc = L.lib().ph_cofacet_rows3(f0.data_ptr(), f1.data_ptr(), f2.data_ptr(), T, E, 100000, off_d.data_ptr(),
                                  too_long, got_off.data_ptr(), got.data_ptr(), st.data_ptr(), ws3.data_ptr(), nb3, s)
    assert rc == 2
