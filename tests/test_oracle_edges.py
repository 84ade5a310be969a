"""The oracle's edge-list entry points, used to check clouds too large for
the oracle's own O(n^2 d) enumeration (the 200,000-point configurations):
  * run_edges on a shuffled edge list restores the reference kernel's
    emission order from (i, j) and gives the same filtration, forest and
    diagrams as run, bit for bit;
  * edge_dsq recomputes the dist^2 bits of given pairs;
  * row_edges returns exactly the edges incident to the listed rows.
Checked on golden cases whose oracle runs are pinned to the reference."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from golden_util import load_golden

CASES = ["n500_d10_t28_h2", "o3_1024_t18", "n2000_d10_t22", "h2_grid3_t2", "sphere3_192_full",
         "clifford200_t14_h2"]


@pytest.mark.parametrize("name", CASES)
def test_edge_list_entry_points_agree_with_the_full_run(name):
    z, meta = load_golden(name)
    p, t, md = z["points"], float(z["t"]), meta["max_dim"]
    ref = oracle.run(p, t, md, fused=True)
    perm = np.random.default_rng(0).permutation(ref["edge_i"].shape[0])
    got = oracle.run_edges(ref["edge_i"][perm], ref["edge_j"][perm], ref["edge_dsq"][perm], p.shape[0], md)
    for k in ("edge_i", "edge_j", "edge_dsq", "mst_idx", "h0", "h1", "h2"):
        assert np.array_equal(np.asarray(ref[k]).view(np.uint8), np.asarray(got[k]).view(np.uint8)), k
    d2 = oracle.edge_dsq(p, ref["edge_i"], ref["edge_j"])
    assert np.array_equal(d2.view(np.uint32), ref["edge_dsq"].view(np.uint32))
    rows = np.unique(np.random.default_rng(1).integers(0, p.shape[0], 7)).astype(np.int32)
    re = oracle.row_edges(p, t, rows)
    got_pairs = set(zip(re["edge_i"].tolist(), re["edge_j"].tolist()))
    m = np.isin(ref["edge_i"], rows) | np.isin(ref["edge_j"], rows)
    assert got_pairs == set(zip(ref["edge_i"][m].tolist(), ref["edge_j"][m].tolist()))


def test_run_edges_rejects_malformed_pairs():
    with pytest.raises(ValueError):
        oracle.run_edges(np.array([3], np.int32), np.array([2], np.int32), np.array([1.0], np.float32), 5, 1)
