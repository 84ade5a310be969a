"""Generate golden fixtures by running the reference implementation on the CPU.

This script is test infrastructure. It imports the reference package
(ot-triton-lab/flash-ph) from the ``src`` directory of a checkout, named with
``--reference PATH`` or the ``FLASHPH_REFERENCE_SRC`` environment variable,
and runs its own code on seeded inputs, writing one ``.npz`` per case into
this directory plus ``manifest.json``, and the reference's ``auto_threshold``
and ``enclosing_radius`` values for the threshold cases into
``thresholds.json``. The GPU box never runs it; the committed fixtures
travel instead.

How the reference is driven (all of it is the reference's own code):

* Edges: ``kernels/edge_kernel.py:152 direct_edge_enumerate`` executed by
  the Triton interpreter (``TRITON_INTERPRET=1``), patched in place of
  ``rips._cpu_edge_enumerate`` (``rips.py:221``) so that ``rips_filtration``
  (``rips.py:98``) runs the direct-difference kernel instead of ``cdist``.
  Under the interpreter the squared distance is the non-fused FP32 chain
  ``acc = acc + diff*diff``.
* H0: ``boruvka.py:17 gpu_boruvka_mst`` and the assembly of
  ``persistence.py:169-192``.
* H1: the body of ``reduce_h1_gpu.py:438 rips_h1_gpu_native`` step by step
  (``_lookup_face_ranks_gpu``, ``_build_cofacet_csr_h1``,
  ``_gpu_apparent_pair_predetect``, ``_prepare_numba_state``, ``_reduce_full``)
  so that the apparent and residual pairs are recorded separately; the final
  rows are checked against a direct call of ``rips_h1_gpu_native``.
* H2 (``max_dim=2``): the reference's public path calls giotto-ph, which is
  not installed. The H2 diagram is assembled from the reference's own
  building blocks instead: ``_numba_utils.py:186 _enumerate_rips_tetrahedra``,
  ``cohomology_general.py:418 compute_global_ranks`` and
  ``cohomology_general.py:622 general_cohomology_reduce`` (H1 first with the
  MST edges skipped, then H2 with the H1 pivots cleared). The H1 diagram of
  that assembly is checked to equal the native H1 diagram as a multiset.

* Thresholds: ``threshold.py:20 auto_threshold`` and ``threshold.py:81
  enclosing_radius`` called on numpy inputs (CPU tensors, fp32 ``cdist``
  tiles), without subsampling.

Run: ``python tests/golden/make_golden.py --reference <checkout>/src [case ...]``
(takes a few minutes); ``--thresholds`` writes only ``thresholds.json``.
"""
from __future__ import annotations

import json
import os
import sys
import time

os.environ.setdefault("TRITON_INTERPRET", "1")
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/flashph_numba_cache")

HERE = os.path.dirname(os.path.abspath(__file__))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from cases import CASES, THRESH_CASES, make_points  # noqa: E402


def _reference_src(argv: list[str]) -> str:
    """The reference checkout's ``src`` directory: ``--reference PATH`` or
    ``FLASHPH_REFERENCE_SRC``."""
    if "--reference" in argv:
        k = argv.index("--reference")
        path = argv[k + 1]
        del argv[k:k + 2]
    else:
        path = os.environ.get("FLASHPH_REFERENCE_SRC", "")
    if not path or not os.path.isdir(os.path.join(path, "flash_ph")):
        raise SystemExit("name the reference's src directory with --reference PATH or FLASHPH_REFERENCE_SRC")
    return path


def _load_reference(src: str):
    sys.path.insert(0, src)
    from flash_ph import rips
    from flash_ph.kernels.edge_kernel import direct_edge_enumerate

    def _direct(pts, n, threshold_sq):
        return direct_edge_enumerate(pts.float().contiguous(), n, threshold_sq, 32)

    rips._cpu_edge_enumerate = _direct
    return rips


def _h1_native_steps(filt, n, mst_idx):
    """Replays reduce_h1_gpu.py:471-604 keeping the intermediate results."""
    from flash_ph import reduce_h1_gpu as R
    from flash_ph.kernels.triangle_kernel import triangle_enumerate

    device = torch.device("cpu")
    E = filt.edge_i.shape[0]
    edge_filt = torch.sqrt(filt.edge_dist_sq)
    mst_mask = torch.zeros(E, dtype=torch.bool)
    if mst_idx.numel() > 0:
        mst_mask[mst_idx] = True
    out = {}
    tri = triangle_enumerate(filt.edge_i, filt.edge_j, filt.vert_adj_ptr,
                             filt.vert_adj_idx, filt.vert_adj_rank, E)
    T = tri[0].shape[0]
    out["T"] = T
    if T == 0:
        return out, tri
    face_ranks = R._lookup_face_ranks_gpu(tri[0], tri[1], tri[2],
                                          filt.edge_i, filt.edge_j, n)
    v0, v1, v2 = tri[0].long(), tri[1].long(), tri[2].long()
    colex = v2 * (v2 - 1) * (v2 - 2) // 6 + v1 * (v1 - 1) // 2 + v0
    perm = colex.argsort(stable=True)
    perm = perm[tri[3][perm].long().argsort(stable=True)]
    tri_global_rank = torch.empty(T, dtype=torch.int32)
    tri_global_rank[perm] = torch.arange(T, dtype=torch.int32) + E
    off, cof = R._build_cofacet_csr_h1(face_ranks, tri_global_rank, E, T, device)
    tri_filt_sorted = edge_filt[tri[3][perm].long()]
    r2f = torch.cat([edge_filt, tri_filt_sorted])
    col_ranks = torch.arange(E, dtype=torch.int32)
    cmf, is_app, ap_b, ap_d, ap_piv = R._gpu_apparent_pair_predetect(
        col_ranks, off, cof, mst_mask, r2f, E + T)
    state = R._prepare_numba_state(col_ranks, off, cof, mst_mask, r2f, cmf, is_app)
    pb, pd, eb = R._reduce_full(*state)
    out.update(
        tri_perm_sorted=tri[3][perm].numpy().astype(np.int32),
        n_apparent=int(is_app.sum()),
        residual=int((~is_app & ~mst_mask).sum()),
        ap_births=ap_b.numpy().astype(np.int32),
        ap_deaths=ap_d.numpy().astype(np.int32),
        res_births=np.asarray(pb, dtype=np.int32),
        res_deaths=np.asarray(pd, dtype=np.int32),
        ess_births=np.asarray(eb, dtype=np.int32),
        cofacet_nnz=int(off[-1]),
    )
    return out, tri


def _h2_from_blocks(filt, tri, mst_idx):
    """H1+H2 diagrams assembled from the reference's own H2 building blocks."""
    from flash_ph._numba_utils import _enumerate_rips_tetrahedra
    from flash_ph.cohomology_general import (compute_global_ranks,
                                             general_cohomology_reduce)

    E = filt.edge_i.shape[0]
    edge_filt = torch.sqrt(filt.edge_dist_sq)
    T = tri[0].shape[0]
    tv0, tv1, tv2, tmr = (x.numpy() for x in tri)
    tets = _enumerate_rips_tetrahedra(
        tv0, tv1, tv2, tmr, filt.vert_adj_ptr.numpy(), filt.vert_adj_idx.numpy(),
        filt.vert_adj_rank.numpy(), T)
    Q = tets[0].shape[0]
    simplices = {
        1: torch.stack([filt.edge_i, filt.edge_j], 1),
        2: torch.stack([tri[0], tri[1], tri[2]], 1),
        3: torch.from_numpy(np.stack(tets[:4], 1)),
    }
    filts = {
        1: edge_filt,
        2: edge_filt[tri[3].long()],
        3: edge_filt[torch.from_numpy(tets[4]).long()] if Q else torch.empty(0),
    }
    granks, r2f = compute_global_ranks(simplices, filts)

    def key(a, b):
        return a.astype(np.int64) * 65536 + b.astype(np.int64)

    # edge -> global rank lookup by vertex pair
    ei = filt.edge_i.numpy(); ej = filt.edge_j.numpy()
    emap = dict(zip(key(ei, ej).tolist(), granks[1].numpy().tolist()))
    tri_rows = [[] for _ in range(T)]
    edge_cof = [[] for _ in range(E)]
    erank_to_idx = {int(g): k for k, g in enumerate(granks[1].numpy().tolist())}
    tg = granks[2].numpy()
    for t in range(T):
        a, b, c = int(tv0[t]), int(tv1[t]), int(tv2[t])
        for (x, y) in ((a, b), (a, c), (b, c)):
            edge_cof[erank_to_idx[emap[x * 65536 + y]]].append(int(tg[t]))
    tmap = {}
    for t in range(T):
        tmap[(int(tv0[t]), int(tv1[t]), int(tv2[t]))] = t
    tri_cof = [[] for _ in range(T)]
    qg = granks[3].numpy() if Q else np.empty(0, np.int32)
    for q in range(Q):
        a, b, c, d = (int(tets[k][q]) for k in range(4))
        for f in ((a, b, c), (a, b, d), (a, c, d), (b, c, d)):
            tri_cof[tmap[f]].append(int(qg[q]))

    def csr(rows):
        off = np.zeros(len(rows) + 1, np.int32)
        off[1:] = np.cumsum([len(r) for r in rows])
        data = np.array([v for r in rows for v in sorted(r)], np.int32)
        return torch.from_numpy(off), torch.from_numpy(data)

    # H1: columns are the edges in rank order (their global ranks)
    e_cols = granks[1]
    off1, cof1 = csr(edge_cof)
    skip1 = torch.zeros(E, dtype=torch.bool)
    if mst_idx.numel() > 0:
        skip1[mst_idx] = True
    pb1, pd1, eb1, piv1 = general_cohomology_reduce(e_cols, off1, cof1, skip1, r2f)
    # H2: columns are triangles (enumeration order), H1 pivots cleared
    off2, cof2 = csr(tri_cof)
    pivset = set(piv1.numpy().tolist())
    skip2 = torch.tensor([int(g) in pivset for g in tg.tolist()], dtype=torch.bool)
    pb2, pd2, eb2, _ = general_cohomology_reduce(granks[2], off2, cof2, skip2, r2f)

    def dgm(pb, pd, eb):
        rows = [(float(r2f[b]), float(r2f[d])) for b, d in zip(pb.tolist(), pd.tolist())]
        rows += [(float(r2f[b]), float("inf")) for b in eb.tolist()]
        return np.array(rows, np.float32).reshape(-1, 2)

    return dgm(pb1, pd1, eb1), dgm(pb2, pd2, eb2), Q


def _sorted_rows(a):
    a = np.asarray(a, np.float32).reshape(-1, 2)
    if a.shape[0] == 0:
        return a
    idx = np.lexsort((a[:, 1], a[:, 0]))
    return a[idx]


def run_case(rips, case):
    from flash_ph.boruvka import gpu_boruvka_mst
    from flash_ph.persistence import rips_persistence
    from flash_ph.reduce_h1_gpu import rips_h1_gpu_native

    pts = make_points(case)
    n = pts.shape[0]
    t = float(case["t"])
    max_dim = int(case["max_dim"])
    res = {"points": pts, "t": np.float64(t)}
    tp = torch.from_numpy(pts)
    filt = rips.rips_filtration(tp, t)
    E = filt.edge_i.shape[0]
    res["edge_i"] = filt.edge_i.numpy().astype(np.int32)
    res["edge_j"] = filt.edge_j.numpy().astype(np.int32)
    res["edge_dsq"] = filt.edge_dist_sq.numpy().astype(np.float32)
    # H0 through the public API (max_dim=0 runs without giotto-ph on CPU)
    h0 = rips_persistence(tp, t, max_dim=0)[0]
    res["h0"] = h0.numpy()
    meta = {"name": case["name"], "n": n, "d": int(pts.shape[1]), "t": t,
            "max_dim": max_dim, "E": E}
    if n <= 1:
        return res, meta
    mst_idx, comp = gpu_boruvka_mst(filt.edge_i, filt.edge_j,
                                    torch.arange(E, dtype=torch.int32), n)
    res["mst_idx"] = mst_idx.numpy().astype(np.int64)
    meta["n_components"] = int(comp.unique().numel())
    if max_dim >= 1:
        h1 = rips_h1_gpu_native(filt, n, mst_idx, t, torch.device("cpu"), backend="gpu")
        res["h1"] = h1.numpy()
        steps, tri = _h1_native_steps(filt, n, mst_idx)
        meta["T"] = int(steps.pop("T"))
        for k in ("n_apparent", "residual", "cofacet_nnz"):
            if k in steps:
                meta[k] = int(steps.pop(k))
        res.update(steps)
    if max_dim >= 2:
        h1b, h2, Q = _h2_from_blocks(filt, tri, mst_idx)
        meta["Q"] = int(Q)
        a = _sorted_rows(res["h1"])
        b = _sorted_rows(h1b)
        assert a.shape == b.shape and np.array_equal(a, b), (
            f"{case['name']}: H1 from blocks differs from native H1")
        res["h2"] = h2
    return res, meta


def make_thresholds():
    """Reference auto_threshold / enclosing_radius values of THRESH_CASES."""
    from flash_ph.threshold import auto_threshold, enclosing_radius

    out = {}
    for case in THRESH_CASES:
        pts = make_points(case)
        out[case["name"]] = {
            "k": case["k"], "percentile": case["percentile"],
            "auto_threshold": float(auto_threshold(pts, k=case["k"], percentile=case["percentile"])),
            "enclosing_radius": float(enclosing_radius(pts)),
        }
        print(case["name"], json.dumps(out[case["name"]]), flush=True)
    with open(os.path.join(HERE, "thresholds.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


def main():
    argv = sys.argv[1:]
    rips = _load_reference(_reference_src(argv))
    if "--thresholds" in argv:
        make_thresholds()
        return
    only = set(argv)
    manifest_path = os.path.join(HERE, "manifest.json")
    manifest = {}
    if os.path.exists(manifest_path):
        with open(manifest_path) as fh:
            manifest = json.load(fh)
    for case in CASES:
        if only and case["name"] not in only:
            continue
        t0 = time.time()
        res, meta = run_case(rips, case)
        meta["generated_s"] = round(time.time() - t0, 2)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **res)
        manifest[case["name"]] = meta
        print(json.dumps(meta), flush=True)
    with open(manifest_path, "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
