"""Proposal network, CPU side: the masks give an autoregressive network, the degree orders the
sampler walks are right, and the FP64 oracle's q is a normalised distribution."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import made_ref


@pytest.mark.parametrize("n,h1,h2", [(8, 16, 24), (16, 32, 32), (512, 1024, 1024)])
def test_masks_are_autoregressive(n, h1, h2):
    from drift_b200.made import masks

    M1, M2, M3 = masks(n, h1, h2)
    R1, R2, R3 = made_ref.masks(n, h1, h2)
    assert np.array_equal(M1, R1) and np.array_equal(M2, R2) and np.array_equal(M3, R3)
    if n <= 16:
        # output i is connected to input j only for j < i, and to every such j through some path
        reach = (M3.astype(np.int64) @ M2 @ M1) > 0
        assert np.array_equal(reach, np.tril(np.ones((n, n), bool), -1))


def test_degree_orders():
    from drift_b200.made import _order, degrees

    n, h = 512, 1024
    d = degrees(n, h)
    ord_, off, most = _order(n, d)
    assert most == 3 and off[-1] == h and off[0] == 0
    for deg in range(1, n + 1):
        units = ord_[off[deg - 1]:off[deg]]
        assert np.all(d[units] == deg)


def test_oracle_q_is_normalised():
    rng = np.random.default_rng(1)
    n, h = 8, 16
    M = made_ref.masks(n, h, h)
    W = [rng.normal(size=m.shape) * m for m in M]
    b = [rng.normal(size=h), rng.normal(size=h), rng.normal(size=n)]
    xs, lq = made_ref.all_logq(W, b, n)
    assert abs(np.exp(lq).sum() - 1.0) < 1e-12
    # the autograd path gives the same log q
    lq2, gW, gb, _ = made_ref.logq_and_grads(W, b, xs[:32])
    assert np.allclose(lq2, lq[:32])
    assert all(g.shape == w.shape for g, w in zip(gW, W))
