"""GUDHI-style RipsComplex wrapper (reference: complex.py)."""
from __future__ import annotations

import numpy as np
import torch

from .persistence import rips_persistence


class RipsComplex:
    """Vietoris-Rips complex whose persistence is computed on the B200.

    Same interface and semantics as the reference's ``complex.py:10-140``:
    intervals come back as float64 numpy arrays, ``persistence()`` as a
    sorted list of ``(dim, (birth, death))``.
    """

    def __init__(self, points, max_edge_length: float):
        if max_edge_length < 0:
            raise ValueError(f"max_edge_length must be non-negative, got {max_edge_length}")
        if isinstance(points, np.ndarray):
            points = torch.from_numpy(points).float()
            if torch.cuda.is_available():
                points = points.cuda()
        self._points = points
        self._max_edge_length = max_edge_length
        self._diagrams = None
        self._max_dim = None

    def compute_persistence(self, max_dim: int = 1, homology_coeff_field: int = 2, backend: str = "auto"):
        """Compute and store the diagrams (returns None, GUDHI convention)."""
        if homology_coeff_field != 2:
            raise ValueError("Only Z/2Z coefficients are supported (homology_coeff_field=2)")
        self._max_dim = max_dim
        self._diagrams = rips_persistence(self._points, self._max_edge_length, max_dim=max_dim,
                                          backend=backend)

    def persistence(self, max_dim: int = 1, homology_coeff_field: int = 2):
        """Compute and return sorted ``(dim, (birth, death))`` pairs.

        The (dim, birth, death) order is made where the diagrams live, with
        stable sorts by death, then birth, then dimension, and the pairs come
        back in one copy (no per-row host work besides building the tuples).
        """
        self.compute_persistence(max_dim, homology_coeff_field)
        live = [(k, d) for k, d in enumerate(self._diagrams) if d.numel() > 0]
        if not live:
            return []
        rows = torch.cat([d.double() for _, d in live])
        dims = torch.cat([torch.full((d.shape[0],), float(k), dtype=torch.float64, device=d.device)
                          for k, d in live])
        order = torch.argsort(rows[:, 1], stable=True)
        order = order[torch.argsort(rows[order, 0], stable=True)]
        order = order[torch.argsort(dims[order], stable=True)]
        table = torch.stack([dims[order], rows[order, 0], rows[order, 1]], dim=1).cpu().tolist()
        return [(int(k), (b, e)) for k, b, e in table]

    def persistence_intervals_in_dimension(self, dim: int):
        """(K, 2) float64 array of the intervals of one dimension."""
        self._check_computed()
        if dim < 0 or dim > self._max_dim:
            return np.empty((0, 2), dtype=np.float64)
        dgm = self._diagrams[dim]
        if dgm.numel() == 0:
            return np.empty((0, 2), dtype=np.float64)
        return dgm.cpu().numpy().astype(np.float64)

    def betti_numbers(self):
        """Number of essential (infinite) classes per dimension."""
        self._check_computed()
        return self._counts(lambda d: d[:, 1] == float("inf"))

    def persistent_betti_numbers(self, from_value: float, to_value: float):
        """Classes born <= from_value and dying > to_value, per dimension."""
        self._check_computed()
        return self._counts(lambda d: (d[:, 0] <= from_value) & (d[:, 1] > to_value))

    def _counts(self, pred):
        # one count per dimension, brought back in one copy
        dev = self._diagrams[0].device
        counts = torch.stack([pred(d).sum() if d.numel() > 0 else torch.zeros((), dtype=torch.int64, device=dev)
                              for d in self._diagrams])
        return [int(c) for c in counts.tolist()]

    def num_vertices(self) -> int:
        return self._points.shape[0]

    def _check_computed(self):
        if self._diagrams is None:
            raise RuntimeError("Call compute_persistence() or persistence() first")
