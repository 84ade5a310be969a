"""Optional CUDA-event timing of named pipeline stages.

Inactive unless a ``record()`` block is open, in which case ``stage(name)``
records a start and an end event on the current stream around the enclosed
launches. Used by the benchmark to time the edge-enumeration kernel inside
the timed region.
"""
from __future__ import annotations

import contextlib

import torch

_active: list | None = None


@contextlib.contextmanager
def record():
    global _active
    prev, _active = _active, []
    try:
        yield _active
    finally:
        _active = prev


@contextlib.contextmanager
def stage(name: str):
    if _active is None:
        yield
        return
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    try:
        yield
    finally:
        b.record()
        _active.append((name, a, b))


def summarize(events) -> dict:
    """name -> (count, total ms); synchronises on the recorded events."""
    out: dict = {}
    for name, a, b in events:
        b.synchronize()
        c, t = out.get(name, (0, 0.0))
        out[name] = (c + 1, t + a.elapsed_time(b))
    return out
