"""CPU check of bench.py's clock sampler against a stand-in nvidia-smi that
prints the queried CSV fields only for the GPU it is asked for (``-i``):
the sampler names its GPU by the selector it is given (a UUID on a GPU box,
since nvidia-smi numbers physical GPUs and ignores CUDA_VISIBLE_DEVICES),
sampling is live before the timed region starts, the summary keeps the
samples taken inside the region, and it falls back to every sample when the
region was too short to see one. NVML is absent or finds no such GPU here,
so the nvidia-smi summary is the one reported."""
from __future__ import annotations

import os
import stat
import time

LINE = "1965, 1965, 512.3, 0x0000000000000000, Not Active, Not Active, Not Active, {cap}"
UUID = "GPU-01234567-89ab-cdef-0123-456789abcdef"


def _fake_smi(tmp_path, period: float, count: int, cap: str = "Not Active", want: str = UUID):
    path = tmp_path / "nvidia-smi"
    path.write_text("#!/bin/bash\n"
                    f"[ \"$1\" = \"-i\" ] && [ \"$2\" = \"{want}\" ] || exit 6\n"
                    f"for i in $(seq {count}); do echo '{LINE.format(cap=cap)}'; sleep {period}; done\n"
                    "sleep 5\n")
    path.chmod(path.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_samples_inside_the_region(tmp_path, monkeypatch):
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, 0.05, 1000) + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(UUID) as c:
        assert c.first >= 1  # live before the region
        time.sleep(0.4)
    s = c.summary()
    assert s["gpu"] == UUID
    assert s["in_region"] and s["samples"] >= 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []


def test_another_gpus_id_gets_no_samples(tmp_path, monkeypatch):
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, 0.05, 1000) + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler("0") as c:  # a physical index, not this GPU's UUID
        time.sleep(0.2)
    s = c.summary()
    assert s["samples"] == 0 and s["sm_mhz"] is None


def test_short_region_falls_back_to_every_sample(tmp_path, monkeypatch):
    import bench
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, 10.0, 1, cap="Active") + os.pathsep + os.environ["PATH"])
    with bench.ClockSampler(UUID) as c:
        time.sleep(0.05)
    s = c.summary()
    assert not s["in_region"] and s["samples"] == 1
    assert s["reasons"] == ["sw_power_cap"]


def test_selector_without_cuda_is_the_index():
    import bench
    import torch
    if not torch.cuda.is_available():
        assert bench.gpu_selector(0) == "0"
