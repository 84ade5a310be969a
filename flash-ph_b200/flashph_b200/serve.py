"""Serving form: continuous batching of rips_persistence requests on one GPU.

``PersistenceServer.submit(points, max_edge_length, max_dim)`` returns a
future. Worker slots (one CUDA stream each, ``slots`` of them) take work from
the queue as soon as they are free, so requests that arrive while others are
on the GPU join the next batch, whose requests run together as one union on
the device:

* a request of at least ``solo_min_points`` points runs alone through the
  native single-cloud call (``ph_rips_persistence``: its stages are sized to
  the one cloud, and a dense request over the triangle limit fails after its
  exact triangle total, before the filtration order is built);
* the smaller requests waiting in the queue are admitted together, in arrival
  order, up to the admission limits (points and candidate pairs of the batch,
  the request count), and run as one disjoint union through the native batch
  call (``ph_rips_persistence_batch``): one library call with four host waits
  for the whole batch. Its first stages are a counting pass: the exact
  per-request edge, triangle and tetrahedron counts decide, on the device
  side of the call, which requests exceed the reference's limits and whether
  the batch fits its simplex budget (a batch over the budget is split by
  those exact counts before any simplex is stored, which bounds the device
  memory of a batch).

Device memory stays resident between batches: every slot allocates from the
device's stream-ordered pool, which keeps its memory for the process (the
library sets the release threshold), and each slot reuses its own stream.

Every result equals what ``rips_persistence`` returns for that request alone,
bit for bit: requests never interact inside a batch. A request over one of the
reference's limits resolves its future with the reference's ValueError.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future

import numpy as np
import torch

from . import _lib as L
from .batch import rips_persistence_batch, worker_stream as slot_stream
from .persistence import rips_persistence


class _Request:
    __slots__ = ("points", "t", "max_dim", "future", "arrival", "done", "n")

    def __init__(self, points, t, max_dim):
        self.points = points
        self.t = float(t)
        self.max_dim = int(max_dim)
        self.future: Future = Future()
        self.arrival = time.perf_counter()
        self.done = None
        self.n = int(points.shape[0]) if hasattr(points, "shape") and len(points.shape) else 0


class PersistenceServer:
    """Continuous batching of ``rips_persistence`` requests.

    Parameters
    ----------
    slots : batches in flight at once, each on its own stream (default 1:
        on the serving stream, two or three slots measured slower, 109 and
        93 against 166 diagrams/s, since the heavy requests' persistent
        kernels each fill the GPU and contend when they run together).
    solo_min_points : requests this large run alone through the single-cloud
        call (default 1024, the best of 1024 and 4096 measured); smaller ones
        are batched.
    max_batch_points, max_batch_pairs, max_batch_requests : admission limits
        of one batch (points, candidate point pairs, requests).
    max_triangles, max_tetrahedra : the reference's per-request limits.
    """

    def __init__(self, device=None, slots: int = 1, solo_min_points: int = 1024,
                 max_batch_points: int = 1 << 18, max_batch_pairs: int = 1 << 32,
                 max_batch_requests: int = 1024, max_triangles: int = 10_000_000,
                 max_tetrahedra: int = 10_000_000):
        if not torch.cuda.is_available():
            raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.solo_min_points = solo_min_points
        self.max_batch_points = max_batch_points
        self.max_batch_pairs = max_batch_pairs
        self.max_batch_requests = max_batch_requests
        self.max_triangles = max_triangles
        self.max_tetrahedra = max_tetrahedra
        self._queue: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()
        self._closed = False
        self.batches = 0
        self.batch_sizes: list[int] = []
        self._workers = [threading.Thread(target=self._worker, args=(i,), daemon=True, name=f"ph-slot-{i}")
                         for i in range(slots)]
        for w in self._workers:
            w.start()

    def submit(self, points, max_edge_length: float, max_dim: int = 1) -> Future:
        """Queue one request; the future resolves to the list of diagrams."""
        req = _Request(points, max_edge_length, max_dim)
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append(req)
            self._cv.notify()
        return req.future

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _admit(self) -> list[_Request]:
        """The next unit of work: the oldest request alone when it is large,
        else the waiting small requests in arrival order up to the limits
        (large ones stay queued for the next free slot)."""
        head = self._queue[0]
        if head.n >= self.solo_min_points:
            return [self._queue.popleft()]
        batch, keep, pts, pairs = [], collections.deque(), 0, 0
        while self._queue and len(batch) < self.max_batch_requests:
            r = self._queue.popleft()
            if r.n >= self.solo_min_points:
                keep.append(r)
                continue
            if batch and (pts + r.n > self.max_batch_points or pairs + r.n * r.n // 2 > self.max_batch_pairs):
                self._queue.appendleft(r)
                break
            batch.append(r)
            pts += r.n
            pairs += r.n * r.n // 2
        self._queue.extendleft(reversed(keep))
        return batch

    def _worker(self, index: int):
        torch.cuda.set_device(self.device)
        # several slots drive their streams concurrently: plain stream order for
        # their launches (dependently launched blocks would hold SMs while waiting)
        if len(self._workers) > 1:
            L.lib().ph_set_dependent_launch(0)
        stream = slot_stream(self.device, index)
        while True:
            with self._cv:
                while not self._queue and not self._closed:
                    self._cv.wait()
                if not self._queue and self._closed:
                    return
                batch = self._admit()
            try:
                with torch.cuda.stream(stream):
                    if len(batch) == 1 and batch[0].n >= self.solo_min_points:
                        r = batch[0]
                        try:
                            res = [rips_persistence(r.points, r.t, max_dim=r.max_dim)]
                        except ValueError as ex:  # the reference's per-call errors
                            res = [ex]
                    else:
                        res = rips_persistence_batch([r.points for r in batch], [r.t for r in batch],
                                                     [r.max_dim for r in batch], self.max_triangles,
                                                     self.max_tetrahedra)
                        # rips_persistence returns a CPU tensor's diagrams on the CPU
                        res = [[d.cpu() for d in out] if not isinstance(out, Exception) and _on_cpu(r.points)
                               else out for r, out in zip(batch, res)]
                stream.synchronize()
            except Exception as ex:  # a failure of the whole batch goes to each request
                res = [ex] * len(batch)
            now = time.perf_counter()
            with self._cv:
                self.batches += 1
                self.batch_sizes.append(len(batch))
            for r, out in zip(batch, res):
                r.done = now
                if isinstance(out, Exception):
                    r.future.set_exception(out)
                else:
                    r.future.set_result(out)


def _on_cpu(points) -> bool:
    return isinstance(points, torch.Tensor) and points.device.type != "cuda"


def latency_percentiles(arrivals, completions, qs=(50, 99)):
    lat = (np.asarray(completions) - np.asarray(arrivals)) * 1e3
    return {f"p{q}": float(np.percentile(lat, q)) for q in qs}
