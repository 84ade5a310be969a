"""Autotuner of the edge-enumeration kernel for batches of clouds.

Two kernels enumerate the same edges with the same dist^2 bits: the direct
FP32 kernel (128 x 128 point tiles on the CUDA cores) and the tensor-core
screened kernel (128 x 256 BF16 Gram tiles, then an exact FP32 recompute of
the candidates). Which is faster depends on the dimension (the screen's K is
16 * ceil((d + 4) / 16) whatever d is), on the cloud sizes (a tile of a small
cloud is mostly padding) and on the density (every candidate the screen
passes is recomputed). ``choose`` keys a batch on its largest d and the log2
bucket of its mean points per cloud, times both kernels once on the first
batch of each key (CUDA events, the faster of two runs each) and keeps the
winner for the process; the edges per point measured on that batch (the
graph density, known only once the edges exist) are recorded beside the
choice in ``table()``. Results never depend on the choice: both kernels give
the same edge set and bits. ``FLASHPH_EDGE_SCREEN=on`` / ``off`` bypasses the
tuner.
"""
from __future__ import annotations

import math
import threading

import numpy as np
import torch

_LOCK = threading.Lock()
_CHOICE: dict[tuple, int] = {}   # key -> edge mode (1 screened, 2 direct)
_TIMES: dict[tuple, tuple] = {}  # key -> (screened ms, direct ms, edges per point)

SCREEN_MAX_D = 252


def key_for(segs_np: np.ndarray) -> tuple:
    """(largest d, log2 bucket of the mean points per cloud)."""
    k = max(int(segs_np.shape[0]), 1)
    max_d = int(segs_np["d"].max()) if segs_np.shape[0] else 1
    mean_n = float(segs_np["n"].sum()) / k
    return (max_d, int(math.floor(math.log2(max(mean_n, 1.0)))))


def choose(segs_np: np.ndarray, trial) -> int:
    """Edge mode (1 screened, 2 direct) for a batch with this segment table.
    ``trial(screen)`` runs the batch's edge enumeration with the screened
    (True) or direct (False) kernel and returns its edge count; it is called
    only for a key not seen before."""
    key = key_for(segs_np)
    if key[0] > SCREEN_MAX_D:
        return 2
    with _LOCK:
        if key in _CHOICE:
            return _CHOICE[key]
    times, count = {}, 0
    for screen in (True, False):
        best = float("inf")
        for _ in range(2):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            count = trial(screen)
            b.record()
            b.synchronize()
            best = min(best, a.elapsed_time(b))
        times[screen] = best
    mode = 1 if times[True] <= times[False] else 2
    with _LOCK:
        _CHOICE[key] = mode
        _TIMES[key] = (times[True], times[False], count / max(float(segs_np["n"].sum()), 1.0))
    return mode


def table() -> dict:
    """Measurements so far: key -> (screened ms, direct ms, edges per point, mode)."""
    with _LOCK:
        return {k: (*_TIMES[k], _CHOICE[k]) for k in _TIMES}


def reset() -> None:
    with _LOCK:
        _CHOICE.clear()
        _TIMES.clear()
