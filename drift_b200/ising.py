"""Ising models accepted by the engine.

``IsingModel`` keeps the semantics of drift/ising.py:24-78 (dense J symmetrised as (J + J^T)/2 with
a zero diagonal, E(s) = -1/2 s.J.s - h.s, dE_i = 2 s_i (J_i.s + h_i)), so a model built for the
reference is accepted unchanged. ``SparseIsingModel`` holds the same energy as a CSR, for sizes
where the reference's dense float64 J cannot exist (a 3-D L=64 lattice would need 550 GB).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class IsingModel:
    """Dense classical Ising model; see drift/ising.py:24-78."""

    J: np.ndarray
    h: np.ndarray

    def __post_init__(self) -> None:
        self.J = np.asarray(self.J, dtype=np.float64)
        self.h = np.asarray(self.h, dtype=np.float64)
        if self.h.ndim != 1:
            raise ValueError("h must be a 1-D field vector")
        n = self.h.shape[0]
        if self.J.shape != (n, n):
            raise ValueError(f"J must be ({n}, {n}) to match h, got {self.J.shape}")
        self.J = 0.5 * (self.J + self.J.T)
        np.fill_diagonal(self.J, 0.0)

    @property
    def n(self) -> int:
        return self.h.shape[0]

    def energy(self, s: np.ndarray) -> float:
        s = np.asarray(s, dtype=np.float64)
        return float(-0.5 * s @ self.J @ s - self.h @ s)

    def energy_batch(self, S: np.ndarray) -> np.ndarray:
        S = np.asarray(S, dtype=np.float64)
        return -0.5 * np.einsum("mi,ij,mj->m", S, self.J, S, optimize=True) - S @ self.h

    def delta_energy_flip(self, s: np.ndarray, i: int) -> float:
        return float(2.0 * s[i] * (self.J[i] @ s + self.h[i]))

    def local_fields(self, s: np.ndarray) -> np.ndarray:
        return self.J @ s + self.h

    @property
    def nbonds(self) -> int:
        return int(np.count_nonzero(np.triu(self.J)))

    def csr(self):
        """(row_ptr, col_idx, weight) of the non-zero couplings, as drift/gpu.py:71-76 builds them."""
        rows, cols = np.nonzero(self.J)
        weight = self.J[rows, cols].astype(np.float32)
        row_ptr = np.zeros(self.n + 1, dtype=np.int32)
        row_ptr[1:] = np.cumsum(np.bincount(rows, minlength=self.n))
        return row_ptr, cols.astype(np.int32), weight


class SparseIsingModel:
    """Ising model stored as a symmetric CSR (no dense J). Same energy convention as IsingModel.

    Built from undirected edges (i, j, w) with i != j; duplicate edges are summed.
    """

    def __init__(self, n: int, edges_i, edges_j, weights, h=None):
        self._n = int(n)
        i = np.asarray(edges_i, dtype=np.int64)
        j = np.asarray(edges_j, dtype=np.int64)
        w = np.asarray(weights, dtype=np.float64)
        if i.shape != j.shape or i.shape != w.shape:
            raise ValueError("edge arrays must have the same shape")
        if np.any(i == j):
            raise ValueError("self-couplings are not allowed")
        if i.size and (min(i.min(), j.min()) < 0 or max(i.max(), j.max()) >= n):
            raise ValueError("edge index out of range")
        self.h = np.zeros(n, dtype=np.float64) if h is None else np.asarray(h, dtype=np.float64)
        if self.h.shape != (n,):
            raise ValueError(f"h must have shape ({n},)")
        rows = np.concatenate([i, j])
        cols = np.concatenate([j, i])
        vals = np.concatenate([w, w])
        key = rows * n + cols
        order = np.argsort(key, kind="stable")
        key, vals = key[order], vals[order]
        uniq, start = np.unique(key, return_index=True)
        vals = np.add.reduceat(vals, start) if vals.size else vals
        keep = vals != 0.0
        uniq, vals = uniq[keep], vals[keep]
        r = (uniq // n).astype(np.int64)
        self._col = (uniq % n).astype(np.int32)
        self._w = vals
        self._row_ptr = np.zeros(n + 1, dtype=np.int64)
        self._row_ptr[1:] = np.cumsum(np.bincount(r, minlength=n))

    @property
    def n(self) -> int:
        return self._n

    @property
    def nnz(self) -> int:
        return int(self._col.size)

    def csr(self):
        return self._row_ptr.astype(np.int32), self._col, self._w.astype(np.float32)

    def local_fields_nofield(self, s: np.ndarray) -> np.ndarray:
        s = np.asarray(s, dtype=np.float64)
        rows = np.repeat(np.arange(self._n), np.diff(self._row_ptr))
        return np.bincount(rows, weights=self._w * s[self._col], minlength=self._n)

    def energy(self, s: np.ndarray) -> float:
        s = np.asarray(s, dtype=np.float64)
        return float(-0.5 * s @ self.local_fields_nofield(s) - self.h @ s)

    def energy_batch(self, S: np.ndarray) -> np.ndarray:
        return np.array([self.energy(s) for s in np.atleast_2d(S)])

    def delta_energy_flip(self, s: np.ndarray, i: int) -> float:
        a, b = self._row_ptr[i], self._row_ptr[i + 1]
        return float(2.0 * s[i] * (self._w[a:b] @ np.asarray(s, dtype=np.float64)[self._col[a:b]] + self.h[i]))

    def to_dense(self) -> IsingModel:
        J = np.zeros((self._n, self._n))
        rows = np.repeat(np.arange(self._n), np.diff(self._row_ptr))
        J[rows, self._col] = self._w
        return IsingModel(J, self.h.copy())


def model_csr(model):
    """(n, row_ptr, col_idx, weight f32, h f32) for any model with .csr() or a dense .J."""
    if hasattr(model, "csr"):
        row_ptr, col_idx, weight = model.csr()
    else:  # a reference drift.ising.IsingModel (dense J): the CSR of drift/gpu.py:71-76
        Jm = np.ascontiguousarray(model.J, dtype=np.float64)
        rows, cols = np.nonzero(Jm)
        weight = Jm[rows, cols].astype(np.float32)
        row_ptr = np.zeros(model.n + 1, dtype=np.int32)
        row_ptr[1:] = np.cumsum(np.bincount(rows, minlength=model.n))
        col_idx = cols.astype(np.int32)
    h = np.ascontiguousarray(model.h, dtype=np.float32)
    return int(model.n), np.ascontiguousarray(row_ptr, np.int32), np.ascontiguousarray(col_idx, np.int32), \
        np.ascontiguousarray(weight, np.float32), h
