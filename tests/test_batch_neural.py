"""Batched neural proposals, CPU side: padded 2-D EA instances keep every energy, the uneven batch
is reproducible, and the networks' widths respect the sampler's bounds."""

from __future__ import annotations

import numpy as np
import pytest

from drift_b200.batch_neural import MAX_NET_SPINS, default_hidden
from drift_b200.instances import ea2d_batch, ea_2d, ea_2d_padded


@pytest.mark.parametrize("L", [4, 5, 8, 9, 13, 48])
def test_padding_adds_uncoupled_spins_only(L):
    a, b = ea_2d(L, 7), ea_2d_padded(L, 7)
    assert b.n % 8 == 0 and 0 <= b.n - a.n < 8 and b.nnz == a.nnz
    rng = np.random.default_rng(L)
    for _ in range(5):
        s = rng.choice([-1.0, 1.0], size=b.n)
        assert b.energy(s) == a.energy(s[: a.n])
    Jb = b.to_dense().J
    assert np.all(Jb[a.n:] == 0) and np.array_equal(Jb[: a.n, : a.n], a.to_dense().J)


def test_uneven_batch_is_reproducible():
    x, y = ea2d_batch(16, 6), ea2d_batch(16, 6)
    assert [m.n for m in x] == [m.n for m in y]
    assert all(np.array_equal(p.csr()[1], q.csr()[1]) for p, q in zip(x, y))
    sizes = np.array([m.n for m in ea2d_batch(256, 6)])
    assert sizes.min() >= 64 and sizes.max() <= 2304 and np.all(sizes % 8 == 0)


@pytest.mark.parametrize("n", [8, 16, 64, 200, 512])
def test_default_hidden_width(n):
    h = default_hidden(n)
    assert h % 8 == 0 and 8 <= h <= 1024 and h <= 4 * (n - 1) and n <= MAX_NET_SPINS
