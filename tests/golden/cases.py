"""Seeded point-cloud cases shared by the fixture generator and the tests.

The shapes, thresholds and generators restate the reference's own test and
benchmark inputs (``testing/test_persistence.py``, ``testing/test_reduce_h1.py``,
``bench/bench_standard.py:44-70``, ``bench_clifford_torus.py:77-84``), with
numpy ``default_rng`` seeds so that the same points are produced on any host.
"""
from __future__ import annotations

import numpy as np


def gaussian(n, d, seed):
    return np.random.default_rng(seed).standard_normal((n, d)).astype(np.float32)


def circle(n, noise, seed):
    rng = np.random.default_rng(seed)
    th = np.linspace(0, 2 * np.pi, n, endpoint=False)
    pts = np.column_stack([np.cos(th), np.sin(th)])
    if noise:
        pts = pts + rng.standard_normal(pts.shape) * noise
    return pts.astype(np.float32)


def sphere(n, d, seed, noise=0.0):
    rng = np.random.default_rng(seed)
    pts = rng.standard_normal((n, d)).astype(np.float32)
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    if noise:
        pts = pts + (rng.standard_normal(pts.shape) * noise).astype(np.float32)
    return pts.astype(np.float32)


def clifford(n, seed, noise=0.0):
    """Clifford torus (cos t, sin t, cos s, sin s)/sqrt(2) (+ Gaussian noise)."""
    rng = np.random.default_rng(seed)
    t = rng.uniform(0, 2 * np.pi, n)
    s = rng.uniform(0, 2 * np.pi, n)
    pts = np.column_stack([np.cos(t), np.sin(t), np.cos(s), np.sin(s)]) / np.sqrt(2)
    if noise:
        pts = pts + rng.standard_normal((n, 4)) * noise
    return pts.astype(np.float32)


def o3(n, seed):
    """Points of O(3) flattened to R^9 (QR of Gaussian matrices, sign-fixed)."""
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((n, 3, 3))
    out = np.empty((n, 9), dtype=np.float32)
    for i in range(n):
        q, r = np.linalg.qr(m[i])
        s = np.sign(np.diag(r))
        s[s == 0] = 1.0
        out[i] = (q * s[np.newaxis, :]).ravel()
    return out


def grid3():
    c = [[float(x), float(y), float(z)] for x in range(3) for y in range(3) for z in range(3)]
    return np.array(c, dtype=np.float32)


def make_points(case):
    g = case["gen"]
    a = case.get("args", {})
    if g == "gaussian":
        return gaussian(case["n"], case["d"], case["seed"]) * np.float32(a.get("scale", 1.0))
    if g == "circle":
        return circle(case["n"], a.get("noise", 0.0), case["seed"])
    if g == "sphere":
        return sphere(case["n"], case["d"], case["seed"], a.get("noise", 0.0))
    if g == "clifford":
        return clifford(case["n"], case["seed"], a.get("noise", 0.0))
    if g == "o3":
        return o3(case["n"], case["seed"])
    if g == "grid3":
        return grid3()
    if g == "empty":
        return np.zeros((0, case["d"]), dtype=np.float32)
    raise ValueError(g)


def _c(name, gen, n, d, t, max_dim=1, seed=42, **args):
    return {"name": name, "gen": gen, "n": n, "d": d, "t": t,
            "max_dim": max_dim, "seed": seed, "args": args}


CASES = [
    _c("empty_d3", "empty", 0, 3, 1.0, max_dim=2),
    _c("single_d3", "gaussian", 1, 3, 1.0, max_dim=2),
    _c("two_far", "gaussian", 2, 3, 0.01, max_dim=1),
    _c("no_edges_n50_d3", "gaussian", 50, 3, 1e-10),
    _c("tight_n10_d2", "gaussian", 10, 2, 0.5, scale=0.01),
    _c("n50_d2_t3", "gaussian", 50, 2, 3.0),
    _c("n100_d2_t07", "gaussian", 100, 2, 0.7),
    _c("circle12_t18", "circle", 12, 2, 1.8, noise=0.02),
    _c("circle20_t05", "circle", 20, 2, 0.5),
    _c("circle30_t15", "circle", 30, 2, 1.5),
    _c("small_d2_s42", "gaussian", 30, 2, 1.5, seed=42),
    _c("small_d2_s43", "gaussian", 30, 2, 1.5, seed=43),
    _c("small_d2_s44", "gaussian", 30, 2, 1.5, seed=44),
    _c("small_d4_s42", "gaussian", 25, 4, 2.0, seed=42),
    _c("small_d4_s43", "gaussian", 25, 4, 2.0, seed=43),
    _c("small_d10", "gaussian", 20, 10, 3.0),
    _c("d10_n40_t4", "gaussian", 40, 10, 4.0),
    _c("d50_n30_t10", "gaussian", 30, 50, 10.0),
    _c("h2_n30_d3_t2", "gaussian", 30, 3, 2.0, max_dim=2),
    _c("h2_n50_d3_t12", "gaussian", 50, 3, 1.2, max_dim=2, seed=123),
    _c("h2_sphere20", "sphere", 20, 3, 2.0, max_dim=2, noise=0.05),
    _c("h2_n100_d3_t15", "gaussian", 100, 3, 1.5, max_dim=2),
    _c("h2_grid3_t2", "grid3", 27, 3, 2.0, max_dim=2),
    _c("h2_sparse_n20", "gaussian", 20, 3, 0.3, max_dim=2),
    _c("clifford200_t06", "clifford", 200, 4, 0.6),
    _c("clifford200_t14_h2", "clifford", 200, 4, 1.4, max_dim=2, noise=0.02),
    _c("o3_200_t18", "o3", 200, 9, 1.8),
    _c("sphere3_192_full", "sphere", 192, 4, 2.001),
    _c("n500_d10_t28_h2", "gaussian", 500, 10, 2.8, max_dim=2),
    _c("n500_d10_t25_h2", "gaussian", 500, 10, 2.5, max_dim=2),
    _c("o3_1024_t18", "o3", 1024, 9, 1.8),
    _c("n2000_d10_t22", "gaussian", 2000, 10, 2.2),
]

CASE_BY_NAME = {c["name"]: c for c in CASES}


def _th(name, gen, n, d, k=20, percentile=95.0, seed=42, **args):
    return {"name": name, "gen": gen, "n": n, "d": d, "t": 0.0, "max_dim": 0, "seed": seed, "args": args,
            "k": k, "percentile": percentile}


# auto_threshold / enclosing_radius cases (threshold.py:20-200): the defaults
# (k=20, 95th percentile), the larger k the reference's docstring recommends
# for tori (k >= 50), k above 64 and d far above the edge kernels' range,
# exact ties on a lattice, and k clamped to n - 1.
THRESH_CASES = [
    _th("th_n500_d10", "gaussian", 500, 10),
    _th("th_n2000_d3", "gaussian", 2000, 3),
    _th("th_n300_d50_k5_p50", "gaussian", 300, 50, k=5, percentile=50.0),
    _th("th_clifford400_k50", "clifford", 400, 4, k=50, noise=0.02),
    _th("th_n1000_d512_k100_p90", "gaussian", 1000, 512, k=100, percentile=90.0, seed=7),
    _th("th_n700_d300_k64_p99", "gaussian", 700, 300, k=64, percentile=99.0, seed=8),
    _th("th_n1500_d8_k200", "gaussian", 1500, 8, k=200, percentile=95.0, seed=9),
    _th("th_grid3_k6_p50", "grid3", 27, 3, k=6, percentile=50.0),
    _th("th_n50_d2_k100", "gaussian", 50, 2, k=100, percentile=75.0, seed=11),
    _th("th_n2_d3", "gaussian", 2, 3, k=20, seed=12),
]
