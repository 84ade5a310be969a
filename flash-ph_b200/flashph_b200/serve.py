"""Serving form: a continuous-batching request loop on one GPU.

``PersistenceServer.submit(points, max_edge_length, max_dim)`` returns a
future. Worker slots (one CUDA stream each) take work from the queue: a
request of at least ``solo_min_points`` points runs alone through the native
pipeline (``ph_rips_persistence``, one library call that waits on the host
four times at most); the small requests at the head of the queue that fit
the admission limits run together as one batch through the batching
pipeline (``batch.rips_persistence_batch``), which spreads a call's fixed
cost over them; a small request with no company runs alone too. Defaults:
one slot and every request native (``solo_min_points=0``). On the serving
stream neither several slots (streams at once) nor batching the small
requests measured faster than one native call at a time, which already keeps
the GPU busy; both remain available as parameters. Admission is by memory, estimated
from the request sizes (points, candidate pairs); the pipelines' own
counting passes enforce the reference's per-call triangle and tetrahedron
caps per request.

Every result equals what ``rips_persistence`` returns for that request
alone, bit for bit: requests never interact inside a batch.
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
    slots : concurrent batches in flight (each on its own stream; default 1).
    max_batch_points : admission limit on the points of one batch.
    max_batch_pairs : admission limit on candidate point pairs of one batch.
    max_batch_requests : admission limit on requests per batch.
    solo_min_points : requests this large run alone (native pipeline, the
        default for all); smaller ones are batched when more than one waits.
    """

    def __init__(self, device=None, slots: int = 1, max_batch_points: int = 1 << 17,
                 max_batch_pairs: int = 1 << 32, max_batch_requests: int = 1024,
                 max_triangles: int = 10_000_000, max_tetrahedra: int = 10_000_000,
                 solo_min_points: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("flashph_b200 computes on a CUDA device; none is available")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.max_batch_points = max_batch_points
        self.max_batch_pairs = max_batch_pairs
        self.max_batch_requests = max_batch_requests
        self.max_triangles = max_triangles
        self.max_tetrahedra = max_tetrahedra
        self.solo_min_points = solo_min_points
        self._queue: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()
        self._closed = False
        self.batches = 0
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
        if self._queue[0].n >= self.solo_min_points:
            return [self._queue.popleft()]
        batch, pts, pairs = [], 0, 0
        while self._queue and len(batch) < self.max_batch_requests:
            r = self._queue[0]
            n = r.n
            if n >= self.solo_min_points:
                break
            if batch and (pts + n > self.max_batch_points or pairs + n * n // 2 > self.max_batch_pairs):
                break
            batch.append(self._queue.popleft())
            pts += n
            pairs += n * n // 2
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
                    if len(batch) == 1:  # a large request, or a small one with no company: one native call
                        r = batch[0]
                        try:
                            res = [rips_persistence(r.points, r.t, max_dim=r.max_dim)]
                        except ValueError as ex:  # the reference's per-call errors
                            res = [ex]
                    else:
                        res = rips_persistence_batch([r.points for r in batch], [r.t for r in batch],
                                                     [r.max_dim for r in batch], self.max_triangles,
                                                     self.max_tetrahedra)
                stream.synchronize()
                self.batches += 1
            except Exception as ex:  # a failure of the whole batch goes to each request
                res = [ex] * len(batch)
            now = time.perf_counter()
            for r, out in zip(batch, res):
                r.done = now
                if isinstance(out, Exception):
                    r.future.set_exception(out)
                else:
                    r.future.set_result(out)


def latency_percentiles(arrivals, completions, qs=(50, 99)):
    lat = (np.asarray(completions) - np.asarray(arrivals)) * 1e3
    return {f"p{q}": float(np.percentile(lat, q)) for q in qs}
