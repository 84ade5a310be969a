"""Benchmark: plain rips_persistence on n=20000 points in d=10 (H0-H2).

Workload: 20000 i.i.d. N(0,1) float32 points in R^10 from seed 42,
max_edge_length=1.4, max_dim=2 (the reference's "20K x 10 H0-H2 ms"
figure). Synthetic data. One step = one full rips_persistence call.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {flashph,reference}]
                  [--workload {plain,batch,serve,precision,profile}] [--case NAME]

The default line also carries a ``serving`` block: a seeded sample of the
serving request stream (n log-uniform in [100, 50000], d in {4, 10, 50},
threshold = 95th percentile of 20-NN distances, H2 for 20% of requests)
served by the continuous-batching server and by plain per-call
rips_persistence: throughput with every request queued at once, and p50/p99
latency under Poisson arrivals at half the plain path's capacity.
``--workload batch`` runs the batching configuration (4096 clouds);
``--workload serve`` runs the serving stream over a rate sweep.
``--workload profile --case NAME --steps K`` runs a fixed workload K times
with no timing (the cases the ncu summaries under profiles/ were captured on).
``--workload precision`` runs the precision configuration (200000 x 50,
max_edge_length 6.0, max_dim 1; ``--n/--d/--t/--max-dim`` override): the
tensor-core screened edge kernel against the direct FP32 kernel, and the
FP64 error of the diagrams.

Prints one JSON line on rank 0. ``value`` is the device-timed ms per call
with the points resident in HBM; ``e2e`` is the same call made through the
public API with a pinned host array (host->device copy of the points and
device->host copy of the diagrams inside the timed region). Under torchrun
every rank runs an independent replica (the path does not shard); times are
the max over ranks. ``--impl reference`` times the CPU oracle (a port of the
reference's algorithm) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "flash-ph_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

N_POINTS, DIM, THRESH, MAX_DIM, SEED = 20000, 10, 1.4, 2, 42
METRIC = "20Kx10 H0-H2 ms"
PUBLISHED_MS = 43.0  # reference README.md:103, A100-80GB
WORKLOAD = ("plain rips_persistence, n=20000 d=10 N(0,1) seed 42, max_edge_length=1.4, "
            "max_dim=2 (H0-H2), Euclidean, strict filtration")


def make_points(seed=SEED):
    return np.random.default_rng(seed).standard_normal((N_POINTS, DIM)).astype(np.float32)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def gpu_selector(local: int) -> str:
    """The nvidia-smi / NVML identifier of torch device ``local``.

    nvidia-smi and NVML number the physical GPUs and ignore
    CUDA_VISIBLE_DEVICES, so a job given, say, physical GPU 5 as cuda:0 must
    name its GPU by UUID, or it reads another GPU's clocks."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:  # no CUDA (CPU tests): the index is all there is
        return str(local)


class NvmlClockPoller:
    """SM clock and clock-event reasons of one GPU read through NVML every
    ``period`` seconds from a host thread, so that a timed region of a few
    milliseconds still holds samples (nvidia-smi samples every 200 ms at
    best). Inactive (no samples) where NVML cannot be loaded."""

    BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, selector: str, period: float = 0.002):
        self.selector = selector
        self.period = period
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._nv = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = (nv.nvmlDeviceGetHandleByUUID(self.selector) if self.selector.startswith("GPU-")
                 else nv.nvmlDeviceGetHandleByIndex(int(self.selector)))
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._nv, self._h = nv, h
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._nv = None
        return self

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
            except Exception:
                return
            time.sleep(self.period)

    def __exit__(self, *a):
        self._stop.set()
        if self._nv is not None:
            self._t.join(timeout=2)
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        sm = [s for s, _ in self.samples]
        reasons = sorted({nm for _, r in self.samples for nm, b in self.BITS.items() if r & b})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sm)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms, plus NVML
    samples every 2 ms, of the GPU named by ``selector`` (its UUID; a
    bare index only where no UUID is known).

    Entering waits (up to 3 s) until nvidia-smi has produced its first sample,
    so that sampling is live when the timed region starts. The summary is the
    NVML samples when there are any (they fall inside the region), else the
    nvidia-smi samples taken inside the region, else every nvidia-smi sample
    when the region was too short to see one; ``smi`` always carries the
    nvidia-smi summary."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, selector):
        self.selector = str(selector)
        self.proc = None
        self.lines: list[str] = []
        self.nvml = NvmlClockPoller(self.selector)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.selector, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.monotonic()
            while not self.lines and self.proc.poll() is None and time.monotonic() - t0 < 3.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        self.first = len(self.lines)
        self.nvml.__enter__()
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        self.nvml.__exit__(*a)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def smi_summary(self):
        inside = self._summary(self.lines[self.first:])
        if inside["samples"]:
            return dict(inside, in_region=True)
        return dict(self._summary(self.lines), in_region=False)

    def summary(self):
        smi = self.smi_summary()
        nv = self.nvml.summary()
        if nv["samples"]:
            out = dict(nv, in_region=True, source="nvml, 2 ms period, inside the timed region")
            out["reasons"] = sorted(set(out["reasons"]) | (set(smi["reasons"]) if smi["in_region"] else set()))
            if out["sm_max_mhz"] is None:
                out["sm_max_mhz"] = smi["sm_max_mhz"]
        else:
            out = dict(smi, source="nvidia-smi, 200 ms period")
        out["gpu"] = self.selector
        out["smi"] = smi
        return out

    @staticmethod
    def _summary(lines):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- serving and batching workloads ------------------------------------------------
def serving_requests(count, seed=7):
    """Seeded sample of the serving stream: n log-uniform in [100, 50000],
    d in {4, 10, 50}, i.i.d. N(0,1) float32, H2 for 20% of requests."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(100), np.log(50000))))
        d = int(rng.choice([4, 10, 50]))
        md = 2 if rng.random() < 0.2 else 1
        reqs.append([rng.standard_normal((n, d)).astype(np.float32), None, md])
    return reqs


def clifford_cloud(n, d, rng):
    th = rng.uniform(0, 2 * np.pi, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    p = np.column_stack([np.cos(th), np.sin(th), np.cos(ph), np.sin(ph)]) / np.sqrt(2)
    p = p + rng.standard_normal((n, 4)) * 0.02
    full = np.zeros((n, max(d, 4)))
    full[:, :4] = p
    q, r = np.linalg.qr(rng.standard_normal((full.shape[1], full.shape[1])))
    q = q * np.sign(np.diag(r))
    return (full @ q.T)[:, :d].astype(np.float32)


def batching_clouds(count, seed=11):
    """Seeded batching configuration: n log-uniform in [64, 4096], d in
    {3, 8, 32}; even clouds i.i.d. N(0,1), odd clouds noisy Clifford tori
    rotated by a random orthogonal matrix (for d = 3 the first three rotated
    coordinates of the 4-D torus are kept)."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(count):
        n = int(np.exp(rng.uniform(np.log(64), np.log(4096))))
        d = int(rng.choice([3, 8, 32]))
        out.append(rng.standard_normal((n, d)).astype(np.float32) if c % 2 == 0 else clifford_cloud(n, d, rng))
    return out


def _thresholds(clouds):
    from flashph_b200.batch import auto_threshold_batch
    return auto_threshold_batch(clouds, k=20, percentile=95.0)


def _plain_stream(reqs, arrivals):
    """Plain per-call rips_persistence, one request after another (each waits
    for its arrival time). Returns completion times, per-request ok flags and
    per-request service times (the call alone, arrival to completion when the
    GPU was idle)."""
    import torch
    from flashph_b200 import rips_persistence
    t0 = time.perf_counter()
    done, ok, service = [], [], []
    for (p, t, md), a in zip(reqs, arrivals):
        wait = t0 + a - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        s0 = time.perf_counter()
        try:
            rips_persistence(p, t, max_dim=md)
            ok.append(True)
        except ValueError:
            ok.append(False)
        torch.cuda.synchronize()
        done.append(time.perf_counter() - t0)
        service.append(time.perf_counter() - s0)
    return np.asarray(done), np.asarray(ok), np.asarray(service)


def _served_stream(reqs, arrivals, slots=None):
    from flashph_b200.serve import PersistenceServer
    t0 = time.perf_counter()
    done = [0.0] * len(reqs)
    futs = []
    kw = {} if slots is None else {"slots": slots}
    with PersistenceServer(**kw) as srv:
        for k, ((p, t, md), a) in enumerate(zip(reqs, arrivals)):
            wait = t0 + a - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            f = srv.submit(p, t, md)
            f.add_done_callback(lambda _f, k=k: done.__setitem__(k, time.perf_counter() - t0))
            futs.append(f)
        ok = []
        for f in futs:
            try:
                f.result(timeout=600)
                ok.append(True)
            except ValueError:
                ok.append(False)
        sizes = list(srv.batch_sizes)
    return np.asarray(done), np.asarray(ok), sizes


def serving_summary(count, rates_rel=(0.5,), seed=7):
    """Served against plain per-call rips_persistence on a seeded sample of the
    serving stream: throughput in completed diagrams per second (requests over
    the reference's limits are answered with its ValueError and are not
    diagrams) with every request queued at once, each request's latency alone
    on an idle GPU through the plain path, and p50/p99 latency under Poisson
    arrivals at rates given relative to the plain path's request capacity."""
    reqs = serving_requests(count, seed)
    thr = _thresholds([r[0] for r in reqs])
    for r, t in zip(reqs, thr):
        r[1] = t
    # warm both paths over the whole request set: the first pass of a request
    # mix grows the device memory pool to its peak (for the served path, the
    # peak of the batches in flight together), a one-time cost of any server
    _plain_stream(reqs, np.zeros(len(reqs)))
    _served_stream(reqs, np.zeros(len(reqs)))
    burst = np.zeros(count)
    # three alternating bursts per path, medians reported (a single burst varies
    # by tens of percent between runs)
    plain_rates, served_rates, plain_req_s, services = [], [], [], []
    for _ in range(3):
        pd, pok, service = _plain_stream(reqs, burst)
        sd, sok, sizes = _served_stream(reqs, burst)
        assert np.array_equal(pok, sok), "served and plain disagree on which requests are over a limit"
        plain_rates.append(int(pok.sum()) / pd.max())
        served_rates.append(int(sok.sum()) / sd.max())
        plain_req_s.append(count / pd.max())
        services.append(service)
    plain_rate = float(np.median(plain_rates))
    served_rate = float(np.median(served_rates))
    single = np.median(np.stack(services), axis=0) * 1e3  # per request, ms
    out = {"requests": count, "diagrams": int(sok.sum()), "over_limit": int(count - sok.sum()),
           "plain_diagrams_per_s": round(plain_rate, 2), "served_diagrams_per_s": round(served_rate, 2),
           "served_over_plain": round(served_rate / plain_rate, 3),
           "bursts": {"plain": [round(x, 1) for x in plain_rates], "served": [round(x, 1) for x in served_rates]},
           "served_batches_burst": len(sizes), "served_batch_sizes": sorted(sizes, reverse=True)[:12],
           "single_request_ms": {"p50": round(float(np.percentile(single, 50)), 3),
                                 "p99": round(float(np.percentile(single, 99)), 3),
                                 "max": round(float(single.max()), 3)},
           "rates": []}
    rng = np.random.default_rng(seed + 1)
    req_rate = float(np.median(plain_req_s))
    for rel in rates_rel:
        lam = rel * req_rate
        arr = np.cumsum(rng.exponential(1.0 / lam, count))
        pd, _, _ = _plain_stream(reqs, arr)
        sd, _, sizes = _served_stream(reqs, arr)
        pl, sl = (pd - arr) * 1e3, (sd - arr) * 1e3
        out["rates"].append({"requests_per_s": round(lam, 2), "rate_rel_plain_capacity": rel,
                             "plain_p50_ms": round(float(np.percentile(pl, 50)), 3),
                             "plain_p99_ms": round(float(np.percentile(pl, 99)), 3),
                             "served_p50_ms": round(float(np.percentile(sl, 50)), 3),
                             "served_p99_ms": round(float(np.percentile(sl, 99)), 3),
                             "served_p99_over_single_p99": round(float(np.percentile(sl, 99)) /
                                                                 out["single_request_ms"]["p99"], 3),
                             "served_batches": len(sizes)})
    return out


def batching_summary(count, prefix=512, seed=11):
    """The batching configuration: diagrams/s of rips_persistence_batch over
    `count` clouds (two timed runs after a warm run, the faster kept) against
    plain per-call rips_persistence on the first `prefix` of them. Completed
    diagrams only (clouds over the reference's limits get its ValueError)."""
    import torch
    from flashph_b200 import rips_persistence
    from flashph_b200.batch import rips_persistence_batch

    clouds = batching_clouds(count, seed)
    thr = _thresholds(clouds)
    rips_persistence_batch(clouds[:64], thr[:64], 1)  # warm
    torch.cuda.synchronize()
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        res = rips_persistence_batch(clouds, thr, 1)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    bt = min(times)
    ok = sum(not isinstance(r, Exception) for r in res)
    m = min(len(clouds), prefix)
    for p, t in zip(clouds[:16], thr[:16]):  # warm the per-call path
        try:
            rips_persistence(p, t, max_dim=1)
        except ValueError:
            pass
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pok = 0
    for p, t in zip(clouds[:m], thr[:m]):
        try:
            rips_persistence(p, t, max_dim=1)
            pok += 1
        except ValueError:
            pass
    torch.cuda.synchronize()
    pt = time.perf_counter() - t0
    return {"workload": "batching: n log-uniform [64,4096], d in {3,8,32}, half N(0,1), half rotated noisy "
                        "Clifford tori, t = 95th pct 20-NN, max_dim=1; host arrays in, device diagrams out",
            "clouds": len(clouds), "diagrams": ok, "over_limit": len(clouds) - ok,
            "batched_diagrams_per_s": round(ok / bt, 2), "batch_seconds": round(bt, 3),
            "batch_runs_s": [round(x, 3) for x in times],
            "plain_per_call": {"clouds": m, "seconds": round(pt, 3), "diagrams": pok,
                               "diagrams_per_s": round(pok / pt, 2)},
            "batched_over_plain": round((ok / bt) / (pok / pt), 3)}


def run_batching(args, rank, local):
    """Batching configuration as its own line."""
    import torch
    torch.cuda.set_device(local)
    out = batching_summary(args.clouds)
    if rank == 0:
        print(json.dumps({"metric": "batched diagrams/s", "value": out["batched_diagrams_per_s"],
                          "unit": "diagrams/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
                          "dtype": "f32", "config": {"workload": out["workload"], "clouds": out["clouds"]},
                          "batching": out}), flush=True)


def _profile_case(case):
    """Workloads the committed ncu summaries were captured on: (points, t,
    max_dim) for a single call, or a callable."""
    rng = np.random.default_rng
    if case == "bench20k":  # the headline workload
        return make_points(), THRESH, MAX_DIM
    if case == "dense1898":  # a dense cloud of the batching configuration's size: 9.8M triangle rows
        return rng(2).standard_normal((1898, 8)).astype(np.float32), 2.701, 1
    if case == "dense_h2_382":  # a dense H2 request of the serving stream (6.1M tetrahedra)
        return rng(4).standard_normal((382, 50)).astype(np.float32), 9.432, 2
    if case == "reject40k":  # a serving request over the triangle limit (2.26e9 triangles)
        return rng(3).standard_normal((40061, 50)).astype(np.float32), 7.946, 1
    if case == "precision200k":  # the precision configuration
        return rng(SEED).standard_normal((200000, 50)).astype(np.float32), 6.0, 1
    raise ValueError(case)


def run_profile(args, rank, local):
    """A fixed workload run --steps times, for ncu captures (no timing)."""
    import torch
    torch.cuda.set_device(local)
    case = args.case
    if case == "knn20k":
        from flashph_b200 import enclosing_radius
        from flashph_b200.threshold import knn_kth_distance
        x = torch.from_numpy(make_points()).cuda()
        for _ in range(args.steps):
            knn_kth_distance(x, 20)
            knn_kth_distance(x, 100)
            enclosing_radius(x)
    elif case == "batch256":
        from flashph_b200.batch import rips_persistence_batch
        clouds = batching_clouds(256)
        thr = _thresholds(clouds)
        xs = [torch.from_numpy(c).cuda() for c in clouds]
        for _ in range(args.steps):
            rips_persistence_batch(xs, thr, 1)
    else:
        from flashph_b200 import rips_persistence
        pts, t, md = _profile_case(case)
        x = torch.from_numpy(pts).cuda()
        for _ in range(args.steps):
            try:
                rips_persistence(x, t, max_dim=md)
            except ValueError:
                pass
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": case, "steps": args.steps}), flush=True)


def run_serving(args, rank, local):
    import torch
    torch.cuda.set_device(local)
    out = serving_summary(args.serving_requests, rates_rel=(0.25, 0.5, 1.0, 2.0))
    if rank == 0:
        print(json.dumps({"metric": "served diagrams/s", "value": out["served_diagrams_per_s"],
                          "unit": "diagrams/s", "higher_is_better": True, "data": "synthetic", "dtype": "f32",
                          "config": {"workload": "serving: n log-uniform [100,50000], d in {4,10,50}, N(0,1), "
                                                 "t = 95th pct 20-NN, H2 for 20%"}, "serving": out}), flush=True)


def _fp64_errors(pts64, filt, dgms):
    """Max |value - FP64 length of its critical edge| per diagram.

    Every finite birth/death value is sqrt_rn(dist^2) of an edge; the FP64
    length of that edge is recomputed from the points. Values shared by
    several edges take the largest error among them (an upper bound)."""
    import torch
    from flashph_b200.rips import edge_filtration_values

    ev = edge_filtration_values(filt.edge_dist_sq)  # ascending (filtration order)
    i, j = filt.edge_i.long(), filt.edge_j.long()
    l64 = torch.empty(ev.shape[0], dtype=torch.float64, device=ev.device)
    for s in range(0, ev.shape[0], 1 << 20):
        e = slice(s, s + (1 << 20))
        l64[e] = (pts64[i[e]] - pts64[j[e]]).pow(2).sum(1).sqrt()
    err = (ev.double() - l64).abs()
    rel = err / l64.clamp_min(1e-300)
    out = {"edges": {"max_abs": float(err.max()) if err.numel() else 0.0,
                     "max_rel": float(rel.max()) if rel.numel() else 0.0}}
    # largest error within each run of equal fp32 values
    uniq, inv = torch.unique_consecutive(ev, return_inverse=True)
    grp = torch.zeros(uniq.shape[0], dtype=torch.float64, device=ev.device).scatter_reduce(
        0, inv, err, reduce="amax")
    for dim, dg in enumerate(dgms):
        v = dg.reshape(-1)
        v = v[torch.isfinite(v) & (v > 0)]
        if v.numel() == 0:
            out[f"H{dim}"] = {"values": 0, "max_abs": 0.0}
            continue
        k = torch.searchsorted(uniq, v).clamp_max(uniq.shape[0] - 1)
        assert bool((uniq[k] == v).all()), "a diagram value is not an edge length"
        out[f"H{dim}"] = {"values": int(v.numel()), "max_abs": float(grp[k].max())}
    return out


def screened_kernel_ms(pts, t, flush, reps=3):
    """Device time of the screened edge launch alone (ph_batch_edges_enumerate_screened,
    as ph_rips_persistence makes it: one cloud, buffers prepared once, no host
    read-back inside the events), median over reps after warm-up."""
    import torch
    from flashph_b200 import _lib as L
    from flashph_b200.rips import _SEG_DTYPE, enumerate_edges, threshold_sq
    n, d = pts.shape
    seg = np.zeros(1, dtype=_SEG_DTYPE)
    seg[0] = (0, 0, 0, n, d, threshold_sq(t), 1)
    segd = torch.from_numpy(seg.view(np.uint8).copy()).to(pts.device)
    nb = (n + 127) // 128
    blk = torch.tensor([0, nb], dtype=torch.int64, device=pts.device)
    cap = max(int(enumerate_edges(pts, t, screen=True)[0].shape[0]), 1)
    ei = torch.empty(cap, dtype=torch.int32, device=pts.device)
    ej, ed = torch.empty_like(ei), torch.empty(cap, dtype=torch.float32, device=pts.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=pts.device)
    stt = torch.zeros(1, dtype=torch.int32, device=pts.device)
    wsb = L.query("ph_edges_screened_workspace_bytes", n, 1, d)
    ws = torch.empty(wsb, dtype=torch.uint8, device=pts.device)
    ntiles = L.query("ph_cloud_tiles", n)
    ts = []
    for _ in range(reps + 3):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        L.call("ph_batch_edges_enumerate_screened", pts.data_ptr(), segd.data_ptr(), 1, ntiles, d, n,
               blk.data_ptr(), nb, ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), cap, cnt.data_ptr(),
               stt.data_ptr(), 0, ws.data_ptr(), wsb, L.stream_handle(pts.device))
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    assert int(stt.item()) == 0
    return statistics.median(ts[3:])


def tc_mma_flops(n, d):
    """MMA flops the screened kernel issues: 2 x 128 x 128 x 16*ceil((d+4)/16)
    per 128 x 128 point tile, nt(nt+1)/2 tiles."""
    nt = (n + 127) // 128
    return 2.0 * 128 * 128 * (((d + 4 + 15) // 16) * 16) * nt * (nt + 1) / 2


def precision_summary(dev, n, d, t, md, steps, warmup, seed=SEED, clock_sel=None):
    """Precision form on n x d N(0,1) points: the screened edge kernel against
    the direct FP32 kernel (identical edge sets required), the tensor-core
    roofline of the screened launch alone, the full call device-timed (L2
    flushed) and end to end, and the FP64 error of the diagrams' critical edge
    lengths."""
    import torch
    from flashph_b200 import _edges, _lib, _timing, rips_persistence
    from flashph_b200.rips import enumerate_edges, rips_filtration

    pts_np = np.random.default_rng(seed).standard_normal((n, d)).astype(np.float32)
    pts = torch.from_numpy(pts_np).to(dev)
    pinned = torch.from_numpy(pts_np).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            r = fn()
            b.record()
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.mean(ts), r

    def canon(e):
        i, j, dsq = e
        key = i.long() * n + j.long()
        o = torch.argsort(key)
        return key[o], dsq[o].view(torch.int32)

    es = enumerate_edges(pts, t, screen=True, stats=True)
    stats = dict(_edges.last_screen_stats)
    dir_ms, ed = timed(lambda: enumerate_edges(pts, t, screen=False), 3)
    ka, da = canon(es)
    kb, db = canon(ed)
    identical = bool(ka.shape == kb.shape and torch.equal(ka, kb) and torch.equal(da, db))
    kern_ms = screened_kernel_ms(pts, t, flush, reps=max(3, min(steps, 10)))

    for _ in range(max(warmup, 3)):
        rips_persistence(pts, t, max_dim=md)
    torch.cuda.synchronize()
    l0 = _lib.launch_count()
    clocks = None
    with _timing.record() as stages:
        if clock_sel is not None:
            with ClockSampler(clock_sel) as cs:
                ms, out = timed(lambda: rips_persistence(pts, t, max_dim=md), steps)
            clocks = cs.summary()
        else:
            ms, out = timed(lambda: rips_persistence(pts, t, max_dim=md), steps)
    launches = (_lib.launch_count() - l0) // (steps + 1)
    e2e_ms, res = timed(lambda: rips_persistence(pinned, t, max_dim=md), max(3, steps // 2))
    st = _timing.summarize(stages)

    tc_flops = tc_mma_flops(n, d)
    pk, src = peaks()
    bf16_peak = pk.get("bf16_tflops", 1590.0)
    tf = tc_flops / (kern_ms * 1e-3) / 1e12
    filt = rips_filtration(pts, t)
    errs = _fp64_errors(pts.double(), filt, out)
    return {
        "pts_np": pts_np, "ms": ms, "e2e_ms": e2e_ms, "launches": launches, "clocks": clocks,
        "h2d": int(pinned.numel() * 4), "d2h": int(sum(r.numel() * 4 for r in res)),
        "rows": [int(o.shape[0]) for o in out],
        "stages_ms": {k: round(v[1] / max(v[0], 1), 4) for k, v in st.items()},
        "edges": {"E": int(ka.shape[0]), "pairs": n * (n - 1) // 2, "screened_kernel_ms": round(kern_ms, 4),
                  "direct_ms": round(dir_ms, 3), "speedup": round(dir_ms / kern_ms, 2),
                  "identical_to_direct": identical, "screen_candidates": stats["candidates"],
                  "forced_pairs": stats["forced"],
                  "candidates_per_edge": round(stats["candidates"] / max(1, int(ka.shape[0])), 3)},
        "tensor": {"kernel": "k_tc_edges (tensor-core screened edge enumeration, with its prep launches)",
                   "bound": "tensor", "achieved": round(tf, 2), "peak": bf16_peak, "unit": "TFLOP/s",
                   "frac": round(tf / bf16_peak, 4), "algorithmic_flops_per_launch": tc_flops,
                   "avg_launch_ms": round(kern_ms, 4),
                   "per_unit": "2 x 128 x 128 x 16*ceil((d+4)/16) MMA flops per 128x128 point tile, "
                               "nt(nt+1)/2 tiles",
                   "peak_source": f"bf16_tflops burst ({src} peaks file)"},
        "fp64_error": errs,
    }


def precision_block(dev, steps=5, warmup=3):
    """The precision configuration (200000 x 50, t=6.0, H0-H1) as a sub-block
    of the default line."""
    p = precision_summary(dev, 200000, 50, 6.0, 1, steps, warmup)
    return {"workload": "rips_persistence, n=200000 d=50 N(0,1) seed 42, max_edge_length=6.0, max_dim=1",
            "call_ms": round(p["ms"], 3), "e2e_ms": round(p["e2e_ms"], 3),
            "identical_to_direct": p["edges"]["identical_to_direct"], "edges": p["edges"],
            "tensor": p["tensor"], "fp64_error": p["fp64_error"], "rows": p["rows"]}


def run_precision(args, rank, local):
    """Precision form as its own line: rips_persistence on n x d N(0,1)
    points (default 200000 x 50, max_edge_length 6.0, max_dim 1)."""
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, d, t, md = args.n or 200000, args.d or 50, args.t or 6.0, 1 if args.max_dim is None else args.max_dim
    steps = max(3, args.steps)
    p = precision_summary(dev, n, d, t, md, steps, args.warmup, seed=SEED + rank, clock_sel=gpu_selector(local))
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        oracle.build()
        m = min(n, 40000)
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.run(p["pts_np"][:m], t, md, fused=True, nthreads=cores)
        sec = time.perf_counter() - t0
        scale = (n * (n - 1)) / (m * (m - 1))
        cpu = {"value": round(sec * 1e3 * scale, 1), "unit": "ms", "cores": cores, "kind": "port",
               "sample": f"C++ port of the reference algorithm on the first {m} points "
                         f"({sec:.2f} s), scaled by the pair count to n={n}"}
    if rank == 0:
        print(json.dumps({
            "metric": f"{n // 1000}Kx{d} H0-H{md} ms (precision form)", "value": round(p["ms"], 3), "unit": "ms",
            "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3), "higher_is_better": False,
            "dtype": "f32 (bf16 screen)", "data": "synthetic",
            "config": {"workload": f"rips_persistence, n={n} d={d} N(0,1) seed {SEED}, max_edge_length={t}, "
                                   f"max_dim={md}", "l2": "flushed before every timed call (256 MiB write)"},
            "e2e": {"value": round(p["e2e_ms"], 3), "unit": "ms", "h2d_bytes_per_step": p["h2d"],
                    "d2h_bytes_per_step": p["d2h"]},
            "gpu_launches": int(p["launches"]),
            "edges": p["edges"],
            "roofline": dict(p["tensor"], traffic=None),
            "stages_ms": p["stages_ms"],
            "fp64_error": p["fp64_error"],
            "rows": p["rows"],
            "cpu_baseline": cpu, "clocks": p["clocks"]}), flush=True)


def kernel_breakdown(pts, t, max_dim, flush, reps=3):
    """Per-stage device times of the staged pipeline (CUDA events around each
    stage's launches) and of the screened edge kernel alone, plus the sizes
    the algorithmic byte and flop counts need. Runs outside the timed region."""
    import torch
    from flashph_b200 import _timing, rips_persistence
    from flashph_b200.cohomology import enumerate_triangles
    from flashph_b200.rips import enumerate_edges, rips_filtration

    os.environ["FLASHPH_PIPELINE"] = "staged"
    try:
        rips_persistence(pts, t, max_dim=max_dim)
        with _timing.record() as ev:
            for _ in range(reps):
                flush.zero_()
                rips_persistence(pts, t, max_dim=max_dim)
            torch.cuda.synchronize()
        st = _timing.summarize(ev)
    finally:
        os.environ.pop("FLASHPH_PIPELINE", None)
    stages = {k: v[1] / max(v[0], 1) for k, v in st.items()}
    edge_ms = screened_kernel_ms(pts, t, flush, reps=reps)
    filt = rips_filtration(pts, t)
    E = int(filt.edge_i.shape[0])
    T = enumerate_triangles(filt).T if max_dim >= 1 else 0
    return stages, edge_ms, E, T


# DRAM traffic per launch from ncu captures of this workload (profiles/*.md)
NCU_TRAFFIC = {
    "k_tc_edges": {"bytes": 2.288e6, "source": "profiles/k_tc_edges_20k_d10.md"},
    "k_reduce": {"bytes": 0.8535e6, "source": "profiles/k_reduce_20k_d10_h1.md"},
    "k_cluster_sort": {"bytes": 0.389e6, "source": "profiles/k_cluster_sort_20k_d10.md"},
}


def rooflines(stages, edge_ms, n, d, E, T, pk, src):
    """Roofline entries of the three kernels that dominate the call."""
    mma_flops = tc_mma_flops(n, d)
    tf = mma_flops / (edge_ms * 1e-3) / 1e12
    bf16 = pk.get("bf16_tflops", 1590.0)
    hbm = pk.get("hbm_gbs", 6650.0)
    out = {}
    out["edges"] = {"kernel": "k_tc_edges (tensor-core screened edge enumeration, with its 4 prep launches)",
                    "bound": "tensor", "achieved": round(tf, 2), "peak": bf16, "unit": "TFLOP/s",
                    "frac": round(tf / bf16, 4), "traffic": NCU_TRAFFIC["k_tc_edges"]["bytes"],
                    "traffic_source": NCU_TRAFFIC["k_tc_edges"]["source"],
                    "algorithmic_flops_per_launch": mma_flops, "avg_launch_ms": round(edge_ms, 5),
                    "per_unit": "2 x 128 x 128 x 16*ceil((d+4)/16) MMA flops per 128x128 point tile, "
                                "nt(nt+1)/2 tiles", "peak_source": f"bf16_tflops burst ({src} peaks file)"}
    if "sort" in stages:
        byts = 2.0 * 12 * E
        gbs = byts / (stages["sort"] * 1e-3) / 1e9
        out["sort"] = {"kernel": "filtration sort (one fused k_cluster_sort launch: packed keys built on load, "
                                 "8 digit passes, edges rebuilt on store)", "bound": "hbm",
                       "achieved": round(gbs, 2), "peak": hbm, "unit": "GB/s", "frac": round(gbs / hbm, 5),
                       "traffic": NCU_TRAFFIC["k_cluster_sort"]["bytes"],
                       "traffic_source": NCU_TRAFFIC["k_cluster_sort"]["source"],
                       "traffic_note": "the fused filtration sort's launch: the 12 bytes per edge are read "
                                       "once, the passes stay in distributed shared memory",
                       "algorithmic_bytes_per_launch": byts,
                       "avg_launch_ms": round(stages["sort"], 5),
                       "per_unit": "12 bytes (i, j, dist^2) read and written per edge",
                       "peak_source": f"hbm_gbs ({src} peaks file)"}
    if "h1.reduce" in stages:
        byts = 4.0 * (E + 1) + 4.0 * 3 * T + 4.0 * T + 1.0 * E + 8.0 * E + 8.0 * T
        gbs = byts / (stages["h1.reduce"] * 1e-3) / 1e9
        out["h1.reduce"] = {"kernel": "k_reduce (H1, with classify/finish/rows)", "bound": "hbm",
                            "achieved": round(gbs, 3), "peak": hbm, "unit": "GB/s", "frac": round(gbs / hbm, 6),
                            "traffic": NCU_TRAFFIC["k_reduce"]["bytes"],
                            "traffic_source": NCU_TRAFFIC["k_reduce"]["source"],
                            "algorithmic_bytes_per_launch": byts, "avg_launch_ms": round(stages["h1.reduce"], 5),
                            "per_unit": "cofacet CSR (4 B per offset and entry), cmf 4 B and owner word 8 B per "
                                        "triangle, mask 1 B and state/pivot 8 B per edge",
                            "note": "latency-bound: the reduction is a chain of dependent column additions "
                                    "(the oracle's critical path), not a bandwidth problem",
                            "peak_source": f"hbm_gbs ({src} peaks file)"}
    return out


def l2_hop_ns(dev, mib=64, hops=200_000, seed=3):
    """Nanoseconds of one dependent L2 load: a single thread chasing a random
    cycle through a 64 MiB buffer (it fits the 126 MB L2), median of 3 laps."""
    import torch
    from flashph_b200 import _lib as L
    n = (mib << 20) // 4
    perm = np.random.default_rng(seed).permutation(n).astype(np.uint32)
    nxt = np.empty(n, dtype=np.uint32)
    nxt[perm] = np.roll(perm, -1)  # one cycle through every entry
    d = torch.from_numpy(nxt.view(np.int32)).to(dev)
    out = torch.zeros(2, dtype=torch.int64, device=dev)
    laps = []
    for _ in range(3):
        L.call("ph_probe_l2_chase", d.data_ptr(), hops, int(perm[0]), out.data_ptr(), L.stream_handle(dev))
        laps.append(float(out[0].item()) / hops)
    return statistics.median(laps)


def latency_roofline(stage_ms, crit_path, hop_ns):
    """The H1 reduction against its latency bound: the oracle's critical path
    (the longest chain of dependent column additions) times two dependent L2
    loads per addition (the pivot's owner word, then the owning record)."""
    min_ms = crit_path * 2 * hop_ns * 1e-6
    return {"kernel": "k_reduce (H1, with classify/finish/rows)", "bound": "latency",
            "crit_path": int(crit_path), "dependent_l2_loads_per_step": 2, "l2_hop_ns": round(hop_ns, 1),
            "min_ms": round(min_ms, 4), "achieved_ms": round(stage_ms, 4), "frac": round(min_ms / stage_ms, 4),
            "per_unit": "crit_path x 2 x measured dependent L2 load latency (one-thread pointer chase, 64 MiB)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(values, world, device):
    """Each value's maximum over the ranks: the job's time is its slowest
    replica's. The same collective on every rank (any backend)."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def run_reference(args, world, rank):
    """CPU oracle (port of the reference algorithm) on all host threads."""
    if rank != 0:
        return
    import oracle

    oracle.build()
    pts = make_points()
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.run(pts, THRESH, MAX_DIM, fused=True, nthreads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run(pts, THRESH, MAX_DIM, fused=True, nthreads=cores)
        times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": round(ms / PUBLISHED_MS, 4),
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": N_POINTS, "d": DIM, "max_edge_length": THRESH,
                   "max_dim": MAX_DIM},
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "port",
                         "sample": "the full workload per step (C++ port of the reference algorithm, "
                                   "edge enumeration on all cores, reduction serial)"},
        "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 300 for the plain workload, so that the clock sampler sees "
                         "the timed region; 20 otherwise)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("flashph", "reference"), default="flashph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-batching", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=96)
    ap.add_argument("--workload", choices=("plain", "batch", "serve", "precision", "profile"), default="plain")
    ap.add_argument("--case", default="bench20k", help="profile workload: bench20k, dense1898, dense_h2_382, "
                                                        "reject40k, precision200k, knn20k, batch256")
    ap.add_argument("--clouds", type=int, default=4096)
    ap.add_argument("--n", type=int, default=None, help="precision workload: points")
    ap.add_argument("--d", type=int, default=None, help="precision workload: dimension")
    ap.add_argument("--t", type=float, default=None, help="precision workload: max_edge_length")
    ap.add_argument("--max-dim", type=int, default=None, help="precision workload: max_dim")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 300 if args.impl == "flashph" and args.workload == "plain" else 20
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "batch":
        run_batching(args, rank, local)
        return
    if args.workload == "serve":
        run_serving(args, rank, local)
        return
    if args.workload == "precision":
        run_precision(args, rank, local)
        return
    if args.workload == "profile":
        run_profile(args, rank, local)
        return

    import torch
    import torch.distributed as dist

    from flashph_b200 import _lib, _timing, rips_persistence

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    pts_np = make_points(SEED + rank)
    pts = torch.from_numpy(pts_np).to(dev)
    pinned = torch.from_numpy(pts_np).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()

    def step():
        return rips_persistence(pts, THRESH, max_dim=MAX_DIM)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    # device-timed region: points resident in HBM, L2 flushed before every step
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    l0 = _lib.launch_count()
    with ClockSampler(gpu_selector(local)) as clocks, _timing.record() as stages:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            out = step()
            ends[k].record()
        torch.cuda.synchronize()
    barrier()
    launches = (_lib.launch_count() - l0) // args.steps
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = statistics.mean(per)
    st = _timing.summarize(stages)

    # end to end through the public API with host buffers
    e2e_ms = []
    h2d = pinned.numel() * 4
    d2h = 0
    for k in range(max(3, args.steps // 2)):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        res = rips_persistence(pinned, THRESH, max_dim=MAX_DIM)  # CPU in, CPU out
        b.record()
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        d2h = sum(r.numel() * 4 for r in res)
    e2e = statistics.mean(e2e_ms)

    ms, e2e = max_over_ranks([ms, e2e], world, dev)

    if rank == 0:
        pk, src = peaks()
        cs = clocks.summary()
        stage_ms, edge_ms, E, T = kernel_breakdown(pts, THRESH, MAX_DIM, flush)
        rl = rooflines(stage_ms, edge_ms, N_POINTS, DIM, E, T, pk, src)
        leaf = {k: v for k, v in stage_ms.items() if k in ("edges", "sort", "vertex_csr", "h1.triangles",
                                                           "h1.cofacets", "h1.reduce", "h2")}
        dominant = max(leaf, key=leaf.get) if leaf else "edges"
        cpu = None
        if not args.no_cpu_baseline and world == 1:  # the host-core baseline belongs to the one-GPU line
            import oracle

            oracle.build()
            cores = os.cpu_count() or 1
            t0 = time.perf_counter()
            ref = oracle.run(pts_np, THRESH, MAX_DIM, fused=True, nthreads=cores)
            cpu_ms = (time.perf_counter() - t0) * 1e3
            if "h1.reduce" in stage_ms:
                rl["h1.reduce.latency"] = latency_roofline(stage_ms["h1.reduce"], ref["crit_path"], l2_hop_ns(dev))
            cpu = {"value": round(cpu_ms, 2), "unit": "ms", "cores": cores, "kind": "port",
                   "sample": "one run of the full workload (C++ port of the reference algorithm)"}
        rows = [int(o.shape[0]) for o in out]
        line = {
            "metric": METRIC, "value": round(ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": round(ms / PUBLISHED_MS, 5), "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N_POINTS, "d": DIM, "max_edge_length": THRESH,
                       "max_dim": MAX_DIM, "replicas": world,
                       "l2": "flushed before every timed step (256 MiB write)", "rows": rows},
            "e2e": {"value": round(e2e, 4), "unit": "ms", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": dict(rl.get(dominant, rl["edges"]), stage=dominant),
            "rooflines": rl,
            "cpu_baseline": cpu,
            # device time x median SM clock: thousands of SM cycles per step
            "clocks": dict(cs, kcycles_per_step=round(ms * cs["sm_mhz"], 1)) if cs.get("sm_mhz") else cs,
            "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "stages_source": "staged pipeline (the same stages called one by one from Python), CUDA events "
                             "around each stage, 3 calls outside the timed region; the timed calls run the "
                             "native pipeline",
            "sizes": {"edges": E, "triangles": T},
        }
        if not args.no_serving and world == 1:  # one-GPU sub-measurements
            line["serving"] = serving_summary(args.serving_requests, rates_rel=(0.5,))
        if not args.no_precision and world == 1:
            line["precision"] = precision_block(dev)
        if not args.no_batching and world == 1:
            line["batching"] = batching_summary(args.clouds)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
