"""Ising models accepted by the engine.

Energy convention (the interface of drift/ising.py:50-68, which every layer of the engine keeps):
``E(s) = -1/2 s.J.s - h.s`` over a symmetric coupling matrix with a zero diagonal, and the energy
change of flipping spin i is ``2 s_i (J_i.s + h_i)``. A dense matrix given by the caller is made
symmetric by averaging it with its transpose (drift/ising.py:41), so an asymmetric input means what
it means to the reference.

Both model classes share one evaluator (`_IsingEnergy`) that works from coupling fields
``F = J s`` computed for a whole batch of configurations at once: ``DenseIsingModel`` computes them
with one matrix product, ``SparseIsingModel`` from its CSR without ever forming J (a 3-D L = 64
lattice would need a 550 GB dense float64 matrix). Objects of the reference's own ``IsingModel``
class are accepted unchanged wherever the engine takes a model (`model_csr` reads only ``.J``,
``.h`` and ``.n``).
"""

from __future__ import annotations

import numpy as np


def _dense_csr(J: np.ndarray, n: int):
    """(row_ptr, col_idx, weight f32) of the non-zero entries of a dense J in row-major order.

    Row-major order is the order drift/gpu.py:71-76 writes the CSR in; the greedy colouring visits
    neighbours in this order, so keeping it keeps the reference's colouring.
    """
    nz = J != 0.0
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(nz.sum(axis=1), out=row_ptr[1:])
    col_idx = np.nonzero(nz)[1].astype(np.int32)
    return row_ptr, col_idx, J[nz].astype(np.float32)


class _IsingEnergy:
    """Energies of one or many configurations from the coupling fields ``J s`` of a subclass."""

    h: np.ndarray

    @property
    def n(self) -> int:
        return int(self.h.shape[0])

    def coupling_fields(self, S: np.ndarray) -> np.ndarray:  # (m, n) -> (m, n): row k is J @ S[k]
        raise NotImplementedError

    def energy_batch(self, S: np.ndarray) -> np.ndarray:
        S = np.atleast_2d(np.asarray(S, dtype=np.float64))
        return -np.sum(S * (0.5 * self.coupling_fields(S) + self.h), axis=1)

    def energy(self, s: np.ndarray) -> float:
        return float(self.energy_batch(s)[0])

    def local_fields(self, s: np.ndarray) -> np.ndarray:
        return self.coupling_fields(np.atleast_2d(np.asarray(s, dtype=np.float64)))[0] + self.h

    def delta_energy_flip(self, s: np.ndarray, i: int) -> float:
        s = np.asarray(s, dtype=np.float64)
        return float(2.0 * s[i] * self.local_fields(s)[i])


class DenseIsingModel(_IsingEnergy):
    """Ising model with a dense coupling matrix (float64), symmetrised with a zero diagonal."""

    def __init__(self, J, h):
        h = np.array(h, dtype=np.float64)
        J = np.array(J, dtype=np.float64)
        if h.ndim != 1:
            raise ValueError(f"the field must be a vector, got an array of shape {h.shape}")
        if J.shape != (h.size, h.size):
            raise ValueError(f"couplings of shape {J.shape} do not match a field of {h.size} spins")
        sym = J + J.T
        sym *= 0.5
        sym[np.diag_indices(h.size)] = 0.0
        self.J = sym
        self.h = h

    def coupling_fields(self, S: np.ndarray) -> np.ndarray:
        return S @ self.J  # J is symmetric

    @property
    def nbonds(self) -> int:
        """Undirected couplings (non-zero entries above the diagonal)."""
        return int(np.count_nonzero(self.J)) // 2

    def csr(self):
        return _dense_csr(self.J, self.n)


# The engine's own dense model under the domain's usual name (the reference's IsingModel objects
# are accepted as they are; see `model_csr`).
IsingModel = DenseIsingModel


class SparseIsingModel(_IsingEnergy):
    """Ising model stored as a symmetric CSR (no dense J), same energy convention.

    Built from undirected edges (i, j, w) with i != j; duplicate edges are summed and couplings that
    sum to zero are dropped.
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

    def coupling_fields(self, S: np.ndarray) -> np.ndarray:
        # per row k: F[k, i] = sum over the CSR entries of row i of w * S[k, col]
        rows = np.repeat(np.arange(self._n), np.diff(self._row_ptr))
        out = np.zeros((S.shape[0], self._n))
        for k in range(S.shape[0]):
            out[k] = np.bincount(rows, weights=self._w * S[k, self._col], minlength=self._n)
        return out

    def local_fields_nofield(self, s: np.ndarray) -> np.ndarray:
        return self.coupling_fields(np.atleast_2d(np.asarray(s, dtype=np.float64)))[0]

    def delta_energy_flip(self, s: np.ndarray, i: int) -> float:
        a, b = self._row_ptr[i], self._row_ptr[i + 1]
        s = np.asarray(s, dtype=np.float64)
        return float(2.0 * s[i] * (self._w[a:b] @ s[self._col[a:b]] + self.h[i]))

    def to_dense(self) -> DenseIsingModel:
        J = np.zeros((self._n, self._n))
        rows = np.repeat(np.arange(self._n), np.diff(self._row_ptr))
        J[rows, self._col] = self._w
        return DenseIsingModel(J, self.h.copy())


def model_csr(model):
    """(n, row_ptr, col_idx, weight f32, h f32) for any model with .csr() or a dense .J."""
    if hasattr(model, "csr"):
        row_ptr, col_idx, weight = model.csr()
    else:  # a reference drift.ising.IsingModel (dense J, already symmetric)
        row_ptr, col_idx, weight = _dense_csr(np.asarray(model.J, dtype=np.float64), int(model.n))
    h = np.ascontiguousarray(model.h, dtype=np.float32)
    return int(model.n), np.ascontiguousarray(row_ptr, np.int32), np.ascontiguousarray(col_idx, np.int32), \
        np.ascontiguousarray(weight, np.float32), h
