"""CPU-only checks: host validation, the C ABI's exported symbols, and the
tie-breaking rule of the filtration sort on the oracle."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest
import torch

import oracle
from flashph_b200 import RipsComplex, rips_persistence
from flashph_b200 import _build
from flashph_b200.rips import threshold_sq

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "flashph_b200.h")


def _declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ph_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    path = _build.build()
    lib = ctypes.CDLL(path)
    syms = _declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.ph_version() == 100


def test_library_is_built_for_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(_build.ARCH_FLAGS)


@pytest.mark.parametrize("kwargs,msg", [
    (dict(max_edge_length=-1.0), "max_edge_length must be non-negative"),
    (dict(max_edge_length=1.0, max_dim=3), "max_dim must be 0, 1, or 2"),
    (dict(max_edge_length=1.0, backend="nope"), "backend must be one of"),
])
def test_validation_messages(kwargs, msg):
    pts = torch.zeros(5, 2)
    with pytest.raises(ValueError, match=msg):
        rips_persistence(pts, **kwargs)


def test_validation_shape_and_h2_limit():
    with pytest.raises(ValueError, match="points must have shape"):
        rips_persistence(torch.zeros(5), 1.0)
    with pytest.raises(ValueError, match="H2 requires n < 65536"):
        rips_persistence(torch.zeros(65536, 2), 1.0, max_dim=2)


def test_trivial_sizes_need_no_device():
    out = rips_persistence(torch.zeros(0, 3), 1.0, max_dim=2)
    assert len(out) == 3 and all(o.shape == (0, 2) for o in out)
    out = rips_persistence(torch.zeros(1, 3), 1.0, max_dim=1)
    assert out[0].tolist() == [[0.0, float("inf")]] and out[1].shape == (0, 2)


def test_ripscomplex_errors_without_compute():
    rc = RipsComplex(torch.zeros(4, 2), 1.0)
    for f in (lambda: rc.persistence_intervals_in_dimension(0), rc.betti_numbers,
              lambda: rc.persistent_betti_numbers(0.0, 1.0)):
        with pytest.raises(RuntimeError, match="compute_persistence"):
            f()
    with pytest.raises(ValueError, match="Z/2Z"):
        rc.compute_persistence(homology_coeff_field=3)
    with pytest.raises(ValueError, match="non-negative"):
        RipsComplex(torch.zeros(4, 2), -1.0)


def test_threshold_sq_matches_oracle():
    for t in (2.8, 1.4, 1.1, 6.0, 0.1, 1e-10):
        assert np.float32(threshold_sq(t)) == oracle.threshold_sq(t)


def colex_collision_cloud(n=110_000, j1=50_000, i1=7, extra=True):
    """Points on a line, all farther apart than 1.5 except designed unit pairs
    whose 32-bit truncated colex indices collide (n > 92682)."""
    c1 = j1 * (j1 - 1) // 2 + i1
    c2 = c1 + (1 << 32)
    j2 = int((1 + np.sqrt(1 + 8 * c2)) // 2)
    while j2 * (j2 - 1) // 2 > c2:
        j2 -= 1
    i2 = c2 - j2 * (j2 - 1) // 2
    assert 0 <= i2 < j2 < n
    x = np.arange(n, dtype=np.float64) * 10.0
    pairs = [(i1, j1), (i2, j2)]
    if extra:  # a third pair with the same truncated colex
        c3 = c1 + (1 << 33)
        j3 = int((1 + np.sqrt(1 + 8 * c3)) // 2)
        while j3 * (j3 - 1) // 2 > c3:
            j3 -= 1
        i3 = c3 - j3 * (j3 - 1) // 2
        if 0 <= i3 < j3 < n:
            pairs.append((i3, j3))
    for a, b in pairs:
        x[b] = x[a] + 1.0
    pts = np.zeros((n, 2), dtype=np.float32)
    pts[:, 0] = x.astype(np.float32)
    return pts, pairs


def emission_key(i, j):
    return ((i >> 5), (j >> 5), i & 31, j & 31)


def test_oracle_orders_colex_collisions_by_emission():
    pts, pairs = colex_collision_cloud(extra=False)
    n = pts.shape[0]
    r = oracle.run(pts, 1.5, 0, stop_after=1, nthreads=0)
    got = list(zip(r["edge_i"].tolist(), r["edge_j"].tolist()))
    want = sorted(pairs, key=lambda p: emission_key(*p))
    assert r["E"] == len(pairs)
    assert got == want
    keys = [((int(np.float32(1.0).view(np.uint32)) << 32) | ((j * (j - 1) // 2 + i) & 0xFFFFFFFF))
            for i, j in got]
    assert len(set(keys)) == 1  # a genuine tie of the packed key


def test_ripscomplex_formats_match_a_host_sort():
    """persistence() orders (dim, (birth, death)) on the diagrams' device with
    one copy back; the result equals a Python sort of every row, ties and
    infinite deaths included, and the Betti counts come back per dimension."""
    inf = float("inf")
    dgms = [torch.tensor([[0.0, 0.5], [0.0, inf], [0.0, 0.25], [0.0, 0.5], [0.0, inf]]),
            torch.tensor([[0.3, 0.4], [0.3, 0.35], [0.1, inf], [0.3, 0.4]]),
            torch.zeros((0, 2))]
    rc = RipsComplex(torch.zeros(3, 2), 1.0)
    rc.compute_persistence = lambda *a, **k: None
    rc._diagrams, rc._max_dim = dgms, 2
    want = sorted((k, (float(b), float(e))) for k, d in enumerate(dgms) for b, e in d.tolist())
    assert rc.persistence(max_dim=2) == want
    assert rc.betti_numbers() == [2, 1, 0]
    assert rc.persistent_betti_numbers(0.3, 0.36) == [4, 3, 0]
