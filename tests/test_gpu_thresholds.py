"""auto_threshold / enclosing_radius on the GPU (threshold.py:20-200).

Pinned two ways on every threshold case (the defaults, k = 50 on a torus,
k > 64, d = 300 and 512, lattice ties, k clamped to n - 1):
  * against an FP64 restatement (oracle.auto_threshold_f64 /
    enclosing_radius_f64) within the rounding bound of the fp32 distance
    chain: relative (d + 8) * 2^-24 (d + 2 roundings of the squared distance,
    halved by the square root, plus the quantile's interpolation);
  * against the reference's own values (tests/golden/thresholds.json, fp32
    cdist on the CPU, which is within 1.2e-7 of FP64 on these cases) within
    that bound plus 4e-7.
The two k-NN forms (top list for k <= 64 at moderate d, radix select for any
k and d) compute the same squared distances in the same order, so where both
apply they agree bit for bit.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest
import torch

import oracle
from cases import THRESH_CASES, make_points

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "thresholds.json")))
U = 2.0 ** -24


def _tol(d):
    return (d + 8) * U


@pytest.mark.parametrize("case", THRESH_CASES, ids=[c["name"] for c in THRESH_CASES])
def test_thresholds_against_fp64_and_reference(case):
    from flashph_b200 import auto_threshold, enclosing_radius
    pts = make_points(case)
    d = pts.shape[1]
    g = GOLDEN[case["name"]]
    got_a = auto_threshold(torch.from_numpy(pts).cuda(), k=case["k"], percentile=case["percentile"])
    got_e = enclosing_radius(torch.from_numpy(pts).cuda())
    want_a = oracle.auto_threshold_f64(pts, case["k"], case["percentile"])
    want_e = oracle.enclosing_radius_f64(pts)
    assert abs(got_a - want_a) <= _tol(d) * abs(want_a), (got_a, want_a)
    assert abs(got_e - want_e) <= _tol(d) * abs(want_e), (got_e, want_e)
    assert abs(got_a - g["auto_threshold"]) <= (_tol(d) + 4e-7) * abs(g["auto_threshold"])
    assert abs(got_e - g["enclosing_radius"]) <= (_tol(d) + 4e-7) * abs(g["enclosing_radius"])
    # numpy input goes through the same path (moved to the current device)
    assert auto_threshold(pts, k=case["k"], percentile=case["percentile"]) == got_a


def test_kth_distances_for_large_k_and_d_elementwise():
    from flashph_b200.threshold import knn_kth_distance
    pts = np.random.default_rng(3).standard_normal((900, 512)).astype(np.float32)
    for k in (1, 64, 100, 899):
        got = knn_kth_distance(torch.from_numpy(pts).cuda(), k).cpu().numpy().astype(np.float64)
        want = oracle.knn_kth_f64(pts, k)
        assert np.all(np.abs(got - want) <= _tol(512) * want), k


def test_top_list_and_radix_select_agree_bit_for_bit():
    """The batched scan with a declared max_d above the top list's shared
    memory limit runs the radix select on every cloud; the single-cloud scan
    of the same clouds (d <= 32, k <= 64) runs the top list."""
    from flashph_b200 import _lib as L
    from flashph_b200.batch import _Batch
    from flashph_b200.threshold import knn_kth_distance
    rng = np.random.default_rng(4)
    clouds = [rng.standard_normal((int(n), int(d))).astype(np.float32)
              for n, d in ((300, 3), (129, 8), (2, 5), (1000, 32), (77, 10))]
    # lattice ties
    clouds.append(np.stack(np.meshgrid(np.arange(5), np.arange(5), np.arange(4)), -1).reshape(-1, 3)
                  .astype(np.float32))
    dev = torch.device("cuda", torch.cuda.current_device())
    b = _Batch([torch.from_numpy(c) for c in clouds], [0.0] * len(clouds), [0] * len(clouds), dev)
    qb = np.zeros(b.k + 1, dtype=np.int64)
    qb[1:] = np.cumsum((b.segs_np["n"].astype(np.int64) + 127) // 128)
    qb_dev = torch.from_numpy(qb).to(dev)
    for k in (1, 7, 20, 64):
        out = torch.empty(b.N, dtype=torch.float32, device=dev)
        L.call("ph_batch_knn_kth", b.pts.data_ptr(), b.segs.data_ptr(), b.k, qb_dev.data_ptr(), int(qb[-1]),
               4096, k, out.data_ptr(), L.stream_handle(dev))
        vb = b.segs_np["vbase"]
        for c, p in enumerate(clouds):
            kk = max(1, min(k, p.shape[0] - 1))
            single = knn_kth_distance(torch.from_numpy(p).cuda(), kk)
            got = out[int(vb[c]): int(vb[c]) + p.shape[0]]
            assert torch.equal(got.view(torch.int32), single.view(torch.int32)), (k, c)
