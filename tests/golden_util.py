"""Helpers for reading the committed golden fixtures and comparing diagrams."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def manifest() -> dict:
    with open(os.path.join(GOLDEN_DIR, "manifest.json")) as fh:
        return json.load(fh)


def golden_cases(max_n: int | None = None) -> list[str]:
    m = manifest()
    return sorted(k for k, v in m.items() if max_n is None or v["n"] <= max_n)


def load_golden(name: str):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    return {k: z[k] for k in z.files}, manifest()[name]


def sorted_rows(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float32).reshape(-1, 2)
    if a.shape[0] == 0:
        return a
    return a[np.lexsort((a[:, 1], a[:, 0]))]
