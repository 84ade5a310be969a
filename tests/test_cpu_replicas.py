"""The multi-GPU form is replicas only (one independent cloud per rank, no
collective on the data path). Its host logic runs here as two gloo ranks on
the CPU: the timings every rank reports are the maximum over the ranks, and
the reference arm runs on rank 0 alone while the other ranks exit without
work."""
from __future__ import annotations

import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    got = bench.max_over_ranks([1.0 + rank, 7.0 - 2 * rank], world, "cpu")
    w, r, _ = bench.dist_setup()

    class Args:
        gpus, steps, warmup = world, 1, 0

    buf = io.StringIO()
    if r != 0:  # rank 0 would time the CPU port of the reference; the others must do nothing
        with redirect_stdout(buf):
            bench.run_reference(Args, w, r)
    dist.barrier()
    q.put((rank, w, got, buf.getvalue()))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, world, got, printed in out:
        assert world == 2
        assert got == [2.0, 7.0]  # max over ranks of (1 + r) and (7 - 2r)
        if rank != 0:
            assert printed == ""
