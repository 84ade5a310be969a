"""The FP64 threshold oracle against the reference's own auto_threshold and
enclosing_radius values (tests/golden/thresholds.json, produced by
tests/golden/make_golden.py from threshold.py:20-200 with fp32 cdist tiles
on the CPU). The reference's fp32 values lie within 2e-7 relative of FP64 on
every case; the GPU tests then hold the CUDA kernels to the FP64 oracle."""
from __future__ import annotations

import json
import os

import pytest

import oracle
from cases import THRESH_CASES, make_points

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "thresholds.json")))


@pytest.mark.parametrize("case", THRESH_CASES, ids=[c["name"] for c in THRESH_CASES])
def test_fp64_thresholds_pin_to_the_reference(case):
    pts = make_points(case)
    g = GOLDEN[case["name"]]
    assert g["k"] == case["k"] and g["percentile"] == case["percentile"]
    a = oracle.auto_threshold_f64(pts, case["k"], case["percentile"])
    e = oracle.enclosing_radius_f64(pts)
    assert abs(a - g["auto_threshold"]) <= 2e-7 * a
    assert abs(e - g["enclosing_radius"]) <= 2e-7 * e


def test_clamping_and_trivial_inputs():
    import numpy as np
    assert oracle.auto_threshold_f64(np.zeros((1, 3))) == 0.0
    assert oracle.enclosing_radius_f64(np.zeros((0, 3))) == 0.0
    pts = np.array([[0.0, 0.0], [3.0, 4.0]])
    assert oracle.auto_threshold_f64(pts, k=20, percentile=250.0) == 5.0  # k -> 1, percentile -> 100
    assert oracle.enclosing_radius_f64(pts) == 5.0
