"""Edge enumeration over a segment table, direct or tensor-core screened.

Both kernels produce the same edges with the same dist^2 bits (the exact
FP32 chain of the reference's compiled kernel); the screened kernel
(tcgen05 BF16 Gram tiles plus a certified bound) skips the exact chain for
pairs that cannot be edges. ``FLASHPH_EDGE_SCREEN`` selects: ``auto``
(default: screen when some cloud has d >= 8), ``on``, ``off``.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from . import _lib as L
from . import _timing

SCREEN_MIN_D = 8
SCREEN_MAX_D = 252


def use_screen(max_d: int) -> bool:
    mode = os.environ.get("FLASHPH_EDGE_SCREEN", "auto").lower()
    if max_d > SCREEN_MAX_D or mode == "off":
        return False
    return mode == "on" or max_d >= SCREEN_MIN_D


# pairs passed by the screen / pairs recomputed without it, of the last screened call
last_screen_stats = {"candidates": 0, "forced": 0}


def enumerate_segments(pts: torch.Tensor, segs_np: np.ndarray, segs_dev: torch.Tensor, ntiles: int, cap: int,
                       screen: bool | None = None, stats: bool = False):
    """Unsorted edges (global vertex ids) of every cloud in the table.

    With ``stats`` the screened kernel's counters are stored in
    ``last_screen_stats`` (one extra device-to-host read)."""
    dev = pts.device
    s = L.stream_handle(dev)
    k = int(segs_np.shape[0])
    N = int(segs_np["n"].sum())
    max_d = int(segs_np["d"].max()) if k else 1
    screen = use_screen(max_d) if screen is None else screen
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if screen:
        nb = (segs_np["n"].astype(np.int64) + 127) // 128
        blk = np.zeros(k + 1, dtype=np.int64)
        blk[1:] = np.cumsum(nb)
        blk_dev = torch.from_numpy(blk).to(dev, non_blocking=True)
        wsb = L.query("ph_edges_screened_workspace_bytes", N, k, max_d)
        ws = L.workspace(wsb, dev)
        st = torch.zeros(2, dtype=torch.int64, device=dev) if stats else None
    for _ in range(2):
        cap = max(int(cap), 1)
        ei = torch.empty(cap, dtype=torch.int32, device=dev)
        ej = torch.empty(cap, dtype=torch.int32, device=dev)
        ed = torch.empty(cap, dtype=torch.float32, device=dev)
        with _timing.stage("edges"):
            if screen:
                L.call("ph_batch_edges_enumerate_screened", pts.data_ptr(), segs_dev.data_ptr(), k, ntiles, max_d,
                       N, blk_dev.data_ptr(), int(blk[-1]), ei.data_ptr(), ej.data_ptr(), ed.data_ptr(), cap,
                       count.data_ptr(), status.data_ptr(), st.data_ptr() if st is not None else 0,
                       ws.data_ptr(), wsb, s)
            else:
                L.call("ph_batch_edges_enumerate", pts.data_ptr(), segs_dev.data_ptr(), k, ntiles, ei.data_ptr(),
                       ej.data_ptr(), ed.data_ptr(), cap, count.data_ptr(), s)
        host = torch.cat([count, status.long()]).cpu()
        if int(host[1]) != 0:
            raise L.PHError("ph_batch_edges_enumerate_screened", int(host[1]))
        E = int(host[0])
        if screen and st is not None:
            c, f = st.tolist()
            last_screen_stats.update(candidates=int(c), forced=int(f))
            st.zero_()
        if E <= cap:
            return ei[:E], ej[:E], ed[:E]
        if E >= 2 ** 31:
            raise ValueError(f"Edge count {E} exceeds int32 range; reduce max_edge_length")
        cap = E
    raise RuntimeError("edge enumeration did not converge")
