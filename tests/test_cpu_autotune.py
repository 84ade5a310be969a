"""The edge-kernel autotuner's bookkeeping on the CPU (no kernels): a key is
tried once (both kernels, twice each), the faster one is kept for every later
batch with the same (largest d, mean cloud size) key, clouds beyond the
screen's d range never go to the screen, and the table records the times and
the density seen."""
from __future__ import annotations

import numpy as np


class _FakeEvent:
    clock = 0.0

    def __init__(self, enable_timing=True):
        self.t = 0.0

    def record(self):
        self.t = _FakeEvent.clock

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return other.t - self.t


def _segs(ns, ds):
    from flashph_b200.batch import SEG_DTYPE
    s = np.zeros(len(ns), dtype=SEG_DTYPE)
    s["n"] = ns
    s["d"] = ds
    return s


def test_tuner_tries_once_and_keeps_the_faster(monkeypatch):
    import torch
    from flashph_b200 import autotune
    monkeypatch.setattr(torch.cuda, "Event", _FakeEvent)
    autotune.reset()
    calls = []

    def trial(screen):
        calls.append(screen)
        _FakeEvent.clock += 1.0 if screen else 3.0  # the screen takes 1 ms, direct 3
        return 500

    assert autotune.choose(_segs([100, 120], [8, 8]), trial) == 1
    assert calls == [True, True, False, False]
    assert autotune.choose(_segs([110, 100], [8, 3]), trial) == 1  # same key: no new trial
    assert len(calls) == 4
    (k, v), = autotune.table().items()
    assert k == (8, 6) and v[0] == 1.0 and v[1] == 3.0 and abs(v[2] - 500 / 220) < 1e-12 and v[3] == 1

    def slow_screen(screen):
        _FakeEvent.clock += 5.0 if screen else 2.0
        return 10

    assert autotune.choose(_segs([3000], [32]), slow_screen) == 2
    assert autotune.choose(_segs([10, 10], [300, 4]), trial) == 2  # d > 252: direct, no trial
    autotune.reset()
    assert autotune.table() == {}
