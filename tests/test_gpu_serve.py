"""Serving form: results served from mixed continuous batches equal the
results of each request alone (bit for bit), and per-request errors come
back through the request's future."""
from __future__ import annotations

import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bits(t):
    return t.cpu().numpy().astype(np.float32).view(np.uint32)


def test_served_results_equal_alone_results():
    from flashph_b200 import rips_persistence
    from flashph_b200.serve import PersistenceServer
    rng = np.random.default_rng(21)
    reqs = []
    for i in range(48):
        n = int(np.exp(rng.uniform(np.log(20), np.log(1500))))
        d = int(rng.choice([4, 10, 50]))
        t = {4: 0.9, 10: 2.4, 50: 7.2}[d]
        md = 2 if (rng.random() < 0.2 and n < 600) else 1
        reqs.append((rng.standard_normal((n, d)).astype(np.float32), t, md))
    with PersistenceServer(slots=2, max_batch_points=4000, solo_min_points=1 << 30) as srv:
        futs = [None] * len(reqs)

        def producer(lo, hi):
            for k in range(lo, hi):
                futs[k] = srv.submit(reqs[k][0], reqs[k][1], reqs[k][2])

        th = [threading.Thread(target=producer, args=(k, k + 12)) for k in range(0, 48, 12)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        served = [f.result(timeout=300) for f in futs]
        assert srv.batches < len(reqs)  # requests were mixed into shared batches
    for (p, t, md), got in zip(reqs, served):
        alone = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=md)
        assert len(got) == len(alone) == md + 1
        for a, b in zip(got, alone):
            assert a.shape == b.shape and np.array_equal(_bits(a), _bits(b))


def test_served_errors_are_per_request():
    from flashph_b200.serve import PersistenceServer
    rng = np.random.default_rng(2)
    ok = rng.standard_normal((80, 3)).astype(np.float32)
    with PersistenceServer(slots=1) as srv:
        f1 = srv.submit(ok, 0.8, 1)
        f2 = srv.submit(ok, -1.0, 1)
        f3 = srv.submit(rng.standard_normal((70000, 2)).astype(np.float32), 0.01, 2)
        assert len(f1.result(timeout=120)) == 2
        with pytest.raises(ValueError, match="non-negative"):
            f2.result(timeout=120)
        with pytest.raises(ValueError, match="H2 requires n < 65536"):
            f3.result(timeout=120)


def test_solo_and_batched_slots_run_concurrently():
    """Three slots on their own streams, large requests alone through the
    native pipeline and small ones batched, clouds of three dimensions (both
    edge kernels) in flight together: every result equals the alone result."""
    from flashph_b200 import rips_persistence
    from flashph_b200.serve import PersistenceServer
    rng = np.random.default_rng(31)
    reqs = []
    for i in range(40):
        n = int(np.exp(rng.uniform(np.log(50), np.log(9000))))
        d = int(rng.choice([4, 10, 50]))
        t = {4: 0.35, 10: 1.3, 50: 6.3}[d]
        reqs.append((rng.standard_normal((n, d)).astype(np.float32), t, 2 if n < 3000 and i % 5 == 0 else 1))
    with PersistenceServer(slots=3, solo_min_points=2000, max_batch_points=6000) as srv:
        futs = [srv.submit(p, t, md) for p, t, md in reqs]
        served = []
        for f in futs:
            try:
                served.append(f.result(timeout=300))
            except ValueError as ex:
                served.append(ex)
    for (p, t, md), got in zip(reqs, served):
        try:
            alone = rips_persistence(torch.from_numpy(p).cuda(), t, max_dim=md)
        except ValueError as ex:
            assert isinstance(got, ValueError) and str(got) == str(ex)
            continue
        assert not isinstance(got, Exception), got
        for a, b in zip(got, alone):
            assert a.shape == b.shape and np.array_equal(_bits(a), _bits(b))
