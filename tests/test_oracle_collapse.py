"""Edge collapse of the flag filtration leaves every diagram unchanged.

The reference computes H2 with giotto-ph's ``ripser_parallel(...,
collapse_edges=True)`` (``persistence.py:48-51``), which first shrinks the flag
filtration by edge collapses. The CUDA path and the oracle reduce the full
filtration instead. These CPU tests run the oracle both ways on every golden
case and on random clouds and require equal H0, H1 and H2 diagrams (as
multisets), which is the property that makes the two H2 paths return the same
diagram.
"""
from __future__ import annotations

import numpy as np
import pytest

from golden_util import golden_cases, load_golden, sorted_rows

import oracle


def _same_diagrams(a, b):
    for k in ("h0", "h1", "h2"):
        assert np.array_equal(sorted_rows(a[k]), sorted_rows(b[k])), k


@pytest.mark.parametrize("name", golden_cases(max_n=4096))
def test_collapse_keeps_every_golden_diagram(name):
    z, meta = load_golden(name)
    a = oracle.run(z["points"], float(z["t"]), meta["max_dim"], fused=False)
    b = oracle.run_collapsed(z["points"], float(z["t"]), meta["max_dim"], fused=False)
    assert b["E_full"] == a["E"]
    assert b["E"] == a["E"] - b["collapse_removed"]
    _same_diagrams(a, b)


@pytest.mark.parametrize("n,d,t,seed", [(60, 3, 0.9, 0), (80, 2, 0.5, 1), (100, 4, 1.6, 2),
                                        (150, 3, 1.0, 3), (200, 10, 3.2, 4), (120, 2, 0.3, 5)])
def test_collapse_keeps_random_diagrams(n, d, t, seed):
    p = np.random.default_rng(seed).standard_normal((n, d)).astype(np.float32)
    a = oracle.run(p, t, 2)
    b = oracle.run_collapsed(p, t, 2)
    _same_diagrams(a, b)
    # the collapse does work on these clouds: edges dropped, fewer triangles
    assert b["collapse_removed"] > 0
    assert b["T"] <= a["T"]


def test_collapse_on_a_tie_heavy_lattice():
    # 4 x 4 x 3 unit lattice: every edge length is 1 or sqrt(2), so most
    # filtration values are tied and the collapse order meets equal values
    g = np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(3)), -1).reshape(-1, 3).astype(np.float32)
    a = oracle.run(g, 1.5, 2)
    b = oracle.run_collapsed(g, 1.5, 2)
    _same_diagrams(a, b)


@pytest.mark.parametrize("name", [c for c in golden_cases(max_n=4096) if load_golden(c)[1]["E"] <= 1000])
def test_collapse_in_dependency_rounds_equals_last_to_first(name):
    """The round form (every edge whose later triangle and certificate edges are
    decided is decided at once, as a kernel would) gives the same slot for every
    edge as the last-to-first order."""
    z, meta = load_golden(name)
    r = oracle.collapse_slots(z["points"], float(z["t"]), fused=False)
    assert np.array_equal(r["slot_seq"], r["slot_rounds"])
    assert (r["collapse_rounds"] > 0) == (r["E_full"] > 0)
    assert r["collapse_rounds"] <= max(r["E_full"], 0)


@pytest.mark.parametrize("name", [c for c in golden_cases(max_n=4096) if load_golden(c)[1]["E"] <= 1500])
def test_relaxed_round_collapse_keeps_every_diagram(name):
    """The relaxed round form (moves resolved by reservations, repeated until
    no edge can move) ends elsewhere than the last-to-first order but is a
    sequence of valid moves too: the same diagrams, at least as many edges
    removed on these fixtures."""
    z, meta = load_golden(name)
    a = oracle.run(z["points"], float(z["t"]), meta["max_dim"], fused=False)
    b = oracle.run_collapsed(z["points"], float(z["t"]), meta["max_dim"], fused=False)
    c = oracle.run_collapsed(z["points"], float(z["t"]), meta["max_dim"], fused=False, relaxed=True)
    _same_diagrams(a, c)
    assert c["E"] <= b["E"]
