"""Seeded instance generators for the engine's workloads.

``random_graph`` and ``maxcut_ising`` restate the reference builders (drift/builders/qubo.py:40-64)
and consume the same NumPy random stream, so ``random_graph(16, 0.5, seed=3)`` is the reference's
graph. The lattice, regular-graph, Erdos-Renyi and Sherrington-Kirkpatrick generators have no
reference counterpart; they produce the synthetic workloads the engine is measured on.
"""

from __future__ import annotations

import numpy as np

from .ising import IsingModel, SparseIsingModel


def random_graph(n: int, p: float = 0.5, seed: int = 0, weighted: bool = False) -> np.ndarray:
    """Erdos-Renyi G(n, p) weight matrix; the draw order of drift/builders/qubo.py:55-64."""
    rng = np.random.default_rng(seed)
    W = np.zeros((n, n))
    if not weighted:
        iu, ju = np.triu_indices(n, k=1)  # row-major (i, j > i): the reference's loop order
        u = rng.random(iu.size)
        sel = u < p
        W[iu[sel], ju[sel]] = 1.0
        W[ju[sel], iu[sel]] = 1.0
        return W
    for i in range(n):
        for j in range(i + 1, n):
            if rng.random() < p:
                w = rng.uniform(0.5, 2.0)
                W[i, j] = W[j, i] = w
    return W


def maxcut_ising(W: np.ndarray) -> IsingModel:
    """MaxCut on weighted adjacency W -> antiferromagnetic Ising J = -W, h = 0 (qubo.py:40-45)."""
    W = np.asarray(W, dtype=np.float64)
    W = 0.5 * (W + W.T)
    np.fill_diagonal(W, 0.0)
    return IsingModel(-W, np.zeros(W.shape[0]))


def ferro_chain(n: int, j: float = 1.0) -> IsingModel:
    J = np.zeros((n, n))
    for i in range(n - 1):
        J[i, i + 1] = J[i + 1, i] = j
    return IsingModel(J=J, h=np.zeros(n))


def pm_spin_glass(n: int, seed: int, field: float = 0.0) -> IsingModel:
    """Complete +-J glass with optional Gaussian field, the draw order of tests/test_parallel_tempering.py:47-55."""
    rng = np.random.default_rng(seed)
    J = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            J[i, j] = J[j, i] = rng.choice([-1.0, 1.0])
    h = rng.normal(scale=field, size=n) if field else np.zeros(n)
    return IsingModel(J=J, h=h)


def ea_2d(L: int, seed: int) -> SparseIsingModel:
    """2-D Edwards-Anderson +-J spin glass on an L x L periodic lattice, J = +-1 with p = 1/2."""
    rng = np.random.default_rng(seed)
    x, y = np.meshgrid(np.arange(L), np.arange(L), indexing="xy")
    site = (x + L * y).ravel()
    right = (((x + 1) % L) + L * y).ravel()
    down = (x + L * ((y + 1) % L)).ravel()
    i = np.concatenate([site, site])
    j = np.concatenate([right, down])
    w = rng.integers(0, 2, size=i.size) * 2.0 - 1.0
    return SparseIsingModel(L * L, i, j, w)


def ea_2d_padded(L: int, seed: int, multiple: int = 8) -> SparseIsingModel:
    """ea_2d(L, seed) with uncoupled spins appended up to a multiple of `multiple` spins. The extra
    spins leave every energy unchanged; a network over all the spins then has a size the proposal
    kernels take (a multiple of 8), and its proposals stay exact."""
    base = ea_2d(L, seed)
    n = -(-base.n // multiple) * multiple
    row_ptr, col, w = base.csr()
    rows = np.repeat(np.arange(base.n), np.diff(row_ptr))
    keep = rows < col
    return SparseIsingModel(n, rows[keep], col[keep], w[keep].astype(np.float64))


def ea2d_batch(n_instances: int, seed: int, L_min: int = 8, L_max: int = 48) -> list:
    """Uneven 2-D EA +-J instances: L_k uniform in [L_min, L_max] from `seed`, couplings of instance
    k from seed k, each padded to a multiple of 8 spins (ea_2d_padded)."""
    rng = np.random.default_rng(seed)
    Ls = rng.integers(L_min, L_max + 1, size=n_instances)
    return [ea_2d_padded(int(L), k) for k, L in enumerate(Ls)]


def ea_3d(L: int, seed: int) -> SparseIsingModel:
    """3-D Edwards-Anderson +-J spin glass on an L^3 periodic lattice."""
    rng = np.random.default_rng(seed)
    idx = np.arange(L ** 3)
    x, y, z = idx % L, (idx // L) % L, idx // (L * L)
    nb = [((x + 1) % L) + L * (y + L * z), x + L * (((y + 1) % L) + L * z), x + L * (y + L * ((z + 1) % L))]
    i = np.concatenate([idx] * 3)
    j = np.concatenate(nb)
    w = rng.integers(0, 2, size=i.size) * 2.0 - 1.0
    return SparseIsingModel(L ** 3, i, j, w)


def random_regular_edges(n: int, d: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Uniform random d-regular simple graph by the configuration model with rejection."""
    if (n * d) % 2:
        raise ValueError("n * d must be even")
    rng = np.random.default_rng(seed)
    for _ in range(10000):
        stubs = rng.permutation(np.repeat(np.arange(n), d))
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        if np.unique(lo.astype(np.int64) * n + hi).size != lo.size:
            continue
        return lo, hi
    raise RuntimeError("no simple d-regular graph found")


def maxcut_3regular(n: int, seed: int) -> SparseIsingModel:
    """MaxCut on a random 3-regular graph as Ising: J = -1 on every edge (maxcut_ising of W = 1)."""
    i, j = random_regular_edges(n, 3, seed)
    return SparseIsingModel(n, i, j, -np.ones(i.size))


def er_gaussian(n: int, mean_degree: float, seed: int, field_sigma: float = 0.1) -> SparseIsingModel:
    """Erdos-Renyi graph G(n, p = mean_degree / (n - 1)) with J ~ N(0, 1) (fp32) and h ~ N(0, field_sigma)."""
    rng = np.random.default_rng(seed)
    pairs = n * (n - 1) // 2
    p = min(1.0, mean_degree / max(n - 1, 1))
    m = int(rng.binomial(pairs, p))
    keys = np.empty(0, dtype=np.int64)
    while keys.size < m:
        k = m - keys.size
        a = rng.integers(0, n, size=2 * k + 16)
        b = rng.integers(0, n, size=2 * k + 16)
        ok = a != b
        lo, hi = np.minimum(a[ok], b[ok]), np.maximum(a[ok], b[ok])
        keys = np.unique(np.concatenate([keys, lo.astype(np.int64) * n + hi]))
    keys = rng.permutation(keys)[:m]
    keys.sort()
    i, j = keys // n, keys % n
    w = rng.standard_normal(m).astype(np.float32).astype(np.float64)
    h = (rng.standard_normal(n) * field_sigma).astype(np.float32).astype(np.float64)
    return SparseIsingModel(n, i, j, w, h)


def sk_model(n: int, seed: int) -> IsingModel:
    """Sherrington-Kirkpatrick: J_ij ~ N(0, 1)/sqrt(n) on the upper triangle, mirrored; h = 0."""
    rng = np.random.default_rng(seed)
    J = np.zeros((n, n))
    iu, ju = np.triu_indices(n, k=1)
    v = (rng.standard_normal(iu.size) / np.sqrt(n)).astype(np.float32).astype(np.float64)
    J[iu, ju] = v
    J[ju, iu] = v
    return IsingModel(J, np.zeros(n))


def gnp_pm(n: int, p: float, seed: int, field: int = 0) -> IsingModel:
    """G(n, p) with +-1 couplings: the edges of random_graph(n, p, seed), a sign per edge in row-major
    edge order from default_rng(seed + 1); with `field`, h_i = +-field from default_rng(seed + 2)."""
    A = random_graph(n, p, seed)
    iu, ju = np.nonzero(np.triu(A, 1))
    signs = np.random.default_rng(seed + 1).integers(0, 2, size=iu.size) * 2.0 - 1.0
    J = np.zeros((n, n))
    J[iu, ju] = signs
    J[ju, iu] = signs
    h = np.zeros(n) if not field else (np.random.default_rng(seed + 2).integers(0, 2, size=n) * 2.0 - 1.0) * field
    return IsingModel(J, h)
