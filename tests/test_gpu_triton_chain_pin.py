"""Pins which dist^2 arithmetic the reference's compiled GPU kernel uses.

The reference enumerates edges with a Triton kernel (kernels/edge_kernel.py
:111-123) that accumulates ``dist_sq += diff * diff`` over the dimensions,
``diff = x[:, None] - y[None, :]``. Whether the compiler fuses the multiply
and add decides the low bits of every dist^2. The reference cannot be run on
the GPU host, so this test compiles a Triton kernel with the same operation
sequence (test infrastructure only; the product has no Triton) and checks
that its bits equal the oracle's fused chain -- the chain the CUDA edge kernel
implements -- and not the unfused one.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

triton = pytest.importorskip("triton")
tl = pytest.importorskip("triton.language")


@triton.jit
def _pair_dist_sq(pts_ptr, out_ptr, n, stride_pn, stride_pd, B: tl.constexpr, D: tl.constexpr):
    I = tl.program_id(0)
    J = tl.program_id(1)
    src = I * B + tl.arange(0, B)
    tgt = J * B + tl.arange(0, B)
    dist_sq = tl.zeros([B, B], dtype=tl.float32)
    for d_idx in range(D):
        x_d = tl.load(pts_ptr + src * stride_pn + d_idx * stride_pd, mask=src < n, other=0.0).to(tl.float32)
        y_d = tl.load(pts_ptr + tgt * stride_pn + d_idx * stride_pd, mask=tgt < n, other=0.0).to(tl.float32)
        diff = x_d[:, None] - y_d[None, :]
        dist_sq += diff * diff
    mask = (src[:, None] < n) & (tgt[None, :] < n)
    tl.store(out_ptr + src[:, None] * n + tgt[None, :], dist_sq, mask=mask)


def test_compiled_reference_chain_is_the_fused_one():
    n, d = 96, 10
    pts = np.random.default_rng(5).standard_normal((n, d)).astype(np.float32)
    dev = torch.from_numpy(pts).cuda()
    out = torch.zeros(n, n, dtype=torch.float32, device="cuda")
    B = 32
    nb = (n + B - 1) // B
    _pair_dist_sq[(nb, nb)](dev, out, n, dev.stride(0), dev.stride(1), B=B, D=d)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    fused = oracle.run(pts, 1e6, 0, fused=True, stop_after=1)
    plain = oracle.run(pts, 1e6, 0, fused=False, stop_after=1)
    assert fused["E"] == plain["E"] == n * (n - 1) // 2
    g = got[fused["edge_i"], fused["edge_j"]].view(np.uint32)
    assert np.array_equal(g, fused["edge_dsq"].view(np.uint32)), "compiled chain is not the fused one"
    gp = got[plain["edge_i"], plain["edge_j"]].view(np.uint32)
    assert not np.array_equal(gp, plain["edge_dsq"].view(np.uint32)), "chains do not differ at this size"
