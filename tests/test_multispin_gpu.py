"""Multispin lattice engine (GPU): words, energies, bests, rung permutation and exchange counts
bit-exact against the multispin oracle; energies equal to a direct recount of the unpacked spins."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

from drift_b200.multispin import Lattice, MsEngine

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def ladder(R, lo, hi):
    return lo * (hi / lo) ** (np.arange(R) / (R - 1))


@pytest.mark.parametrize("dims,L,R,rounds,spr", [(3, 4, 32, 6, 2), (3, 6, 64, 4, 3), (2, 8, 32, 10, 1), (2, 12, 96, 3, 2)])
def test_multispin_matches_oracle(dims, L, R, rounds, spr):
    lat = Lattice.edwards_anderson(dims, L, 7)
    betas = ladder(R, 0.2, 2.0)
    eng = MsEngine(lat, betas, seed=11, sweeps_per_round=spr, instance=3)
    eng.init()
    eng.run(rounds)
    eng.check()
    st = eng.fetch()
    ost = oracle.ms_run(dims, L, lat.jneg, betas, n_rounds=rounds, sweeps_per_round=spr, seed=11, instance=3)
    assert np.array_equal(st["words"], ost.words)
    assert np.array_equal(st["best_words"], ost.best_words)
    assert np.array_equal(st["energy"], ost.energy)
    assert np.array_equal(st["best_energy"], ost.best_energy)
    assert np.array_equal(st["rung_of_slot"], ost.rung_of_slot)
    assert np.array_equal(st["tried"], ost.tried[: R - 1]) and np.array_equal(st["accepted"], ost.accepted[: R - 1])
    assert np.array_equal(lat.energy(st["spins"]).astype(np.int64), st["energy"])
    assert np.array_equal(lat.energy(st["best_spins"]).astype(np.int64), st["best_energy"])


def test_multispin_resume_and_large_lattice_energies():
    lat = Lattice.edwards_anderson(3, 6, 2)
    betas = ladder(32, 0.2, 2.0)
    a = MsEngine(lat, betas, seed=4, sweeps_per_round=2)
    a.init()
    a.run(9)
    b = MsEngine(lat, betas, seed=4, sweeps_per_round=2)
    b.init()
    b.run(4)
    b.run(5)
    a.check()
    b.check()
    x, y = a.fetch(), b.fetch()
    for k in ("words", "best_words", "energy", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(x[k], y[k]), k
    # the 3-D L = 64 lattice: exact energies after a few rounds, 128 replicas
    big = Lattice.edwards_anderson(3, 64, 5)
    e = MsEngine(big, ladder(128, 0.2, 2.0), seed=1, sweeps_per_round=1)
    e.init()
    e.run(3)
    e.check()
    st = e.fetch()
    assert np.array_equal(big.energy(st["spins"][:8]).astype(np.int64), st["energy"][:8])
    assert np.all(st["best_energy"] <= st["energy"])
